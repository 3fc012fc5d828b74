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
    // Header-driven gate evaluation (what the kernels run) for every type,
    // fan-in count 1..3 and input codes.
    for (uint32_t type = 0; type < PDF_NTYPES; type++) {
        if (type == PDF_INPT) continue;
        for (uint32_t nfi = 1; nfi <= 3; nfi++) {
            const uint32_t h = make_rec_header(type, 0, nfi);
            std::printf("flags %u %u %u %u %u\n", type, nfi, (h & RF_MARKF0) ? 1 : 0, (h & RF_INPT) ? 1 : 0,
                        (h & RF_SENS) ? 1 : 0);
            const uint32_t combos = 1u << (2 * nfi);
            for (uint32_t cmb = 0; cmb < combos; cmb++) {
                uint32_t c[3] = {cmb & 3, (cmb >> 2) & 3, (cmb >> 4) & 3};
                uint32_t V, v1, T;
                eval_first(h, (c[0] & 1) << 7, (c[0] >> 1) << 7, V, v1);
                for (uint32_t j = 1; j <= hdr_nfold(h); j++) eval_fold(h, V, v1, (c[j] & 1) << 7, (c[j] >> 1) << 7);
                eval_finish(h, V, v1, T);
                const uint32_t code = ((V >> 7) & 1) | (((T >> 7) & 1) << 1);
                std::printf("gate %u %u %u %u %u %u\n", type, nfi, c[0], c[1], c[2], code);
            }
        }
    }
    // One-pass side-input test (sens_step / sens_result) for AND..NOR with
    // 2..4 fan-ins and every input code combination.
    for (int robust = 0; robust < 2; robust++)
        for (uint32_t type = PDF_AND; type <= PDF_NOR; type++)
            for (uint32_t nfi = 2; nfi <= 4; nfi++)
                for (uint32_t cmb = 0; cmb < (1u << (2 * nfi)); cmb++) {
                    const bool or_like = type == PDF_OR || type == PDF_NOR;
                    SensAcc s;
                    sens_init(s);
                    for (uint32_t x = 0; x < nfi; x++) {
                        const uint32_t c = (cmb >> (2 * x)) & 3;
                        if (robust)
                            sens_step<1>(s, or_like, (c & 1) << 9, (c >> 1) << 9);
                        else
                            sens_step<0>(s, or_like, (c & 1) << 9, (c >> 1) << 9);
                    }
                    const uint32_t r = robust ? sens_result<1>(s) : sens_result<0>(s);
                    std::printf("sensall %d %u %u %u %u\n", robust, type, nfi, cmb, (r >> 9) & 1);
                }
    // FIXED semantics: header-driven evaluation with true n-input gates, and
    // the one-pass side test with per-fan-in marks, for AND..XNOR with 1..4
    // fan-ins, every code combination and every mark pattern.
    for (uint32_t type = PDF_AND; type <= PDF_XNOR; type++)
        for (uint32_t nfi = 1; nfi <= 4; nfi++) {
            const uint32_t h = make_rec_header(type, 0, nfi, true);
            std::printf("fflags %u %u %u %u %u\n", type, nfi, (h & RF_MARKF0) ? 1 : 0, (h & RF_MANY) ? 1 : 0,
                        (h & RF_SENS) ? 1 : 0);
            for (uint32_t cmb = 0; cmb < (1u << (2 * nfi)); cmb++) {
                uint32_t V, v1, T;
                eval_first(h, (cmb & 1) << 3, ((cmb >> 1) & 1) << 3, V, v1);
                for (uint32_t j = 1; j <= hdr_nfold(h); j++) {
                    const uint32_t c = (cmb >> (2 * j)) & 3;
                    eval_fold<true>(h, V, v1, (c & 1) << 3, (c >> 1) << 3);
                }
                eval_finish<true>(h, V, v1, T);
                std::printf("fgate %u %u %u %u\n", type, nfi, cmb, ((V >> 3) & 1) | (((T >> 3) & 1) << 1));
                if (nfi < 2) continue;
                const uint32_t mor = flagmask(h, RF_IM), mxor = flagmask(h, RF_XOR), mand = ~(mor | mxor);
                for (int nonrobust = 0; nonrobust < 2; nonrobust++)
                    for (uint32_t marks = 0; marks < (1u << nfi); marks++) {
                        SensAcc s;
                        sens_init(s);
                        for (uint32_t x = 0; x < nfi; x++) {
                            const uint32_t c = (cmb >> (2 * x)) & 3, m = ((marks >> x) & 1) << 11;
                            if (nonrobust)
                                sens_step_fixed<1>(s, mand, mor, mxor, (c & 1) << 11, (c >> 1) << 11, m);
                            else
                                sens_step_fixed<0>(s, mand, mor, mxor, (c & 1) << 11, (c >> 1) << 11, m);
                        }
                        const uint32_t r = nonrobust ? sens_result<1>(s) : sens_result<0>(s);
                        std::printf("fsens %d %u %u %u %u %u\n", nonrobust, type, nfi, cmb, marks, (r >> 11) & 1);
                    }
            }
        }
    return 0;
}
