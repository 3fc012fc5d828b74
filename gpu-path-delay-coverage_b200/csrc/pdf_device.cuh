// pdf_device.cuh -- device-side types and bit-plane gate algebra.
//
// A (net, pair) carries the reference's 2-bit transition code
// (bit0 = value under vector 2, bit1 = the value changed).  Here 32 pairs
// share a word: plane V holds bit0 and plane T holds bit1 of 32 codes.  The
// value under vector 1 is V ^ T.  Every reference lookup table is an exact
// per-vector boolean function, so each table becomes two or three bitwise
// operations on words; tests/test_luts.py proves every entry of every table
// equal to these forms.
#ifndef PDF_DEVICE_CUH
#define PDF_DEVICE_CUH

#include <cstdint>

#include "pdf.h"

#ifdef __CUDACC__
#define PDF_HD __host__ __device__ __forceinline__
#else  // host-only compilers (the LUT identity test builds this header with g++)
#define PDF_HD static inline
#define __align__(n) alignas(n)
#endif

typedef unsigned __int128 pdf_u128;

// Gate record, 32 bytes, one per gate, built at circuit upload.
//   w[0] = type | po << 4 | nfi << 8
//   w[1] = nfo
//   w[2] = edge offset: fan-ins at edges[w2 + j], fan-outs at edges[w2 + nfi + k]
//   w[3..7] = fan-ins 0..4 inline (the rest only in edges[])
struct __align__(16) GateRec {
    uint32_t w[8];
};
static constexpr int kInlineFanins = 5;

PDF_HD uint32_t rec_type(const GateRec &r) { return r.w[0] & 0xFu; }
PDF_HD uint32_t rec_po(const GateRec &r) { return (r.w[0] >> 4) & 1u; }
PDF_HD uint32_t rec_nfi(const GateRec &r) { return (r.w[0] >> 8) & 0xFFu; }

// Two-input fold step val = OP2(val, r) on bit-planes (simkernel.cuh:146 via
// the coalesce_t simLUT, :62-95): AND/NAND/OR/NOR evaluate per vector;
// XOR, XNOR and every other type yield S0 (:89-92).
PDF_HD void fold2(uint32_t type, uint32_t &V, uint32_t &T, uint32_t rV, uint32_t rT) {
    const uint32_t a1 = V ^ T, b1 = rV ^ rT;  // values under vector 1
    uint32_t v2, v1;
    switch (type) {
        case PDF_AND:
            v2 = V & rV;
            v1 = a1 & b1;
            break;
        case PDF_NAND:
            v2 = ~(V & rV);
            v1 = ~(a1 & b1);
            break;
        case PDF_OR:
            v2 = V | rV;
            v1 = a1 | b1;
            break;
        case PDF_NOR:
            v2 = ~(V | rV);
            v1 = ~(a1 | b1);
            break;
        default:
            V = 0;
            T = 0;
            return;
    }
    V = v2;
    T = v2 ^ v1;
}

// NOT (notLUT {S1,S0,T1,T0}, simkernel.cuh:165): flip the value, keep the flag.
PDF_HD void not1(uint32_t &V, uint32_t &T) { V = ~V; (void)T; }

// Sensitisation test LUT_16(LUT[type - 2], on, off) (markkernel.cuh:36-41)
// on 32 (on, off) code pairs at once.  robust selects LUT_R, else LUT_NR.
//   AND/NAND LUT_NR 0x2A00: on=T0 & off in {S1,T1}  |  on=T1 & off=S1
//   AND/NAND LUT_R  0x2200: off=S1
//   OR/NOR   LUT_NR 0x5100: on=T0 & off=S0  |  on=T1 & off in {S0,T0}
//   OR/NOR   LUT_R  0x1100: off=S0
//   XOR/XNOR 0x0000: never
template <int ROBUST>
PDF_HD uint32_t sens(uint32_t type, uint32_t onV, uint32_t onT, uint32_t offV, uint32_t offT) {
    switch (type) {
        case PDF_AND:
        case PDF_NAND:
            return ROBUST ? (onT & offV & ~offT) : (onT & offV & (~onV | ~offT));
        case PDF_OR:
        case PDF_NOR:
            return ROBUST ? (onT & ~offV & ~offT) : (onT & ~offV & (~offT | onV));
        default:
            return 0;
    }
}

// Saturating 128-bit add; sets *ovf on overflow.
PDF_HD pdf_u128 add_sat(pdf_u128 a, pdf_u128 b, bool &ovf) {
    const pdf_u128 r = a + b;
    if (r < a) {
        ovf = true;
        return ~(pdf_u128)0;
    }
    return r;
}

#endif
