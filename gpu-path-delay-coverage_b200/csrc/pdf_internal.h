// pdf_internal.h -- host-side types shared by the library's translation units.
#ifndef PDF_INTERNAL_H
#define PDF_INTERNAL_H

#include <cstdint>
#include <vector>

#include "pdf.h"

struct pdf_netbuf {
    uint32_t n_gates = 0, n_levels = 0;
    std::vector<uint32_t> level_offsets;
    std::vector<uint8_t> type, po;
    std::vector<uint32_t> nfi, nfo;
    std::vector<uint64_t> edge_offset;
    std::vector<uint32_t> edges;
};

#endif
