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

// Batches driven by the serving loop, which keeps one pass in flight while
// it prepares the next (pdf_api.cpp):
//   batch_rebind_on   pdf_batch_rebind whose control-block upload is
//                     enqueued on `stream` (in order before the next pass on
//                     it) instead of waited for; the batch must not be
//                     rebound again before that pass is done
//   batch_pass_async  one pass on `stream`, its control word read back into
//                     the batch's pinned staging after it
//   batch_pass_status the status of that pass, once the stream has passed it
typedef struct CUstream_st *cudaStream_t;
pdf_status batch_rebind_on(pdf_batch *b, const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags,
                           cudaStream_t stream);
pdf_status batch_pass_async(pdf_batch *b, cudaStream_t stream);
pdf_status batch_pass_status(const pdf_batch *b);

#endif
