// Prints the bit-plane gate algebra of pdf_device.cuh for every input code,
// so tests/test_luts.py can compare it with the reference's tables.
#include <cstdio>

#include "pdf_device.cuh"

int main() {
    for (uint32_t type = 0; type < PDF_NTYPES; type++)
        for (uint32_t a = 0; a < 4; a++)
            for (uint32_t b = 0; b < 4; b++) {
                // one pair per word, in bit 5 (any lane must behave the same)
                uint32_t V = (a & 1) << 5, T = (a >> 1) << 5;
                fold2(type, V, T, (b & 1) << 5, (b >> 1) << 5);
                const uint32_t code = ((V >> 5) & 1) | (((T >> 5) & 1) << 1);
                std::printf("fold %u %u %u %u\n", type, a, b, code);
                for (int robust = 0; robust < 2; robust++) {
                    const uint32_t s = robust ? sens<1>(type, a & 1, a >> 1, b & 1, b >> 1)
                                              : sens<0>(type, a & 1, a >> 1, b & 1, b >> 1);
                    std::printf("sens %d %u %u %u %u\n", robust, type, a, b, s & 1);
                }
            }
    for (uint32_t a = 0; a < 4; a++) {
        uint32_t V = a & 1, T = a >> 1;
        not1(V, T);
        std::printf("not %u %u\n", a, (V & 1) | ((T & 1) << 1));
    }
    return 0;
}
