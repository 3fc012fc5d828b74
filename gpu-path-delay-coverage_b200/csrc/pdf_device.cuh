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
//   w[0] = type | po << 4 | RF_* flags (bits 5..7, 16..23) | nfi << 8 | nfold << 24
//   w[1] = nfo
//   w[2] = edge offset: fan-ins at edges[w2 + j], fan-outs at edges[w2 + nfi + k]
//   w[3..6] = where the forward kernel reads fan-ins 0..3 (source words):
//          SRC_PLANE | f   the plane row of gate f in global memory
//          SRC_FAR | s     slot s of the piece's far buffer (prefetched)
//          s               slot s of the shared-memory ring of recent gates
//   w[7] = fan-in 0 (its gate id; 0 without fan-ins)
// Fan-ins past the fourth are read from edges[] (ring or plane row).
struct __align__(16) GateRec {
    uint32_t w[8];
};
static constexpr int kInlineFanins = 4;
static constexpr uint32_t SRC_PLANE = 0x80000000u, SRC_FAR = 0x40000000u, SRC_IDX = 0x3FFFFFFFu;
// Lane kernel (tile of 32 words): w[3..6] hold the fan-in ids, with this bit
// set when the fan-in is a killed gate (RF_KILL: its value is S0 and it never
// marks), whose row is then neither read nor, unless someone else reads it,
// written.
static constexpr uint32_t SRC_ZERO = 0x80000000u;
// Gate records per piece of the lane kernel (staged in shared memory).
static constexpr uint32_t kLaneRecs = 1024;
static constexpr uint32_t kMaxFar = 1024;  // far-buffer slots per piece at most

// Per-gate evaluation flags, derived once from (type, nfi) so that the
// kernels evaluate every gate with the same branch-free instruction sequence
// (simkernel.cuh:111-149, markkernel.cuh:233-264):
enum : uint32_t {
    RF_NOT = 1u << 16,     // fan-in 0 enters inverted (NOT with one fan-in)
    RF_IM = 1u << 17,      // fold inputs inverted: OR/NOR as AND of complements
    RF_OM = 1u << 18,      // each fold step inverts its result (NAND, NOR)
    RF_KILL = 1u << 19,    // the value is S0: a multi-input gate whose fold the
                           // coalesced simLUT sends to 0 (XOR, XNOR, NOT, others)
    RF_SENS = 1u << 20,    // the mark needs the side-input test (AND..XNOR, nfi >= 2)
    RF_MARKF0 = 1u << 21,  // mark = transition & mark of fan-in 0
    RF_INPT = 1u << 22,    // primary input: mark = transition
    RF_SPILL = 1u << 23,   // a later gate reads this gate's plane rows from global memory
                           // (lane kernel: some gate reads its rows at all)
    // true n-input semantics (PDF_MARK_FIXED_*)
    RF_XOR = 1u << 5,      // fold steps are XOR (XOR, XNOR)
    RF_OINV = 1u << 6,     // the folded value is inverted under both vectors (NAND, NOR, XNOR)
    RF_MANY = 1u << 7,     // mark = transition & OR over fan-ins i of (mark(i) & side test for i)
};

PDF_HD uint32_t rec_type(const GateRec &r) { return r.w[0] & 0xFu; }
PDF_HD uint32_t rec_po(const GateRec &r) { return (r.w[0] >> 4) & 1u; }
PDF_HD uint32_t rec_nfi(const GateRec &r) { return (r.w[0] >> 8) & 0xFFu; }
PDF_HD uint32_t hdr_nfold(uint32_t h) { return h >> 24; }

// Header word of a gate (w[0]); `fixed` selects the true n-input semantics
// for AND..XNOR (every other type is evaluated as in the reference).
PDF_HD uint32_t make_rec_header(uint32_t type, uint32_t po, uint32_t nfi, bool fixed = false) {
    uint32_t f = 0, nfold = 0;
    const bool two_input = type >= PDF_AND && type <= PDF_XNOR;
    const bool copy = type == PDF_BUFF || type == PDF_FROM || type == PDF_DFF;
    if (fixed && two_input) {
        if (type == PDF_OR || type == PDF_NOR) f |= RF_IM;
        if (type == PDF_XOR || type == PDF_XNOR) f |= RF_XOR;
        if (type == PDF_NAND || type == PDF_NOR || type == PDF_XNOR) f |= RF_OINV;
        f |= nfi >= 2 ? (RF_SENS | RF_MANY) : RF_MARKF0;
        nfold = nfi - 1;
    } else if (type == PDF_INPT) {
        f |= RF_INPT;
    } else if (copy) {
        f |= RF_MARKF0;  // :126-130 copy fan-in 0; mark follows fan-in 0 (:242-246)
    } else if (nfi >= 2 && !(type >= PDF_AND && type <= PDF_NOR)) {
        f |= RF_KILL;  // the fold step yields 0 (:89-92)
        if (type == PDF_NOT || two_input) f |= RF_MARKF0;
    } else {
        if (type == PDF_NOT) f |= RF_NOT | RF_MARKF0;
        if (two_input) f |= RF_MARKF0;
        if (type == PDF_OR || type == PDF_NOR) f |= RF_IM;
        if (type == PDF_NAND || type == PDF_NOR) f |= RF_OM;
        if (two_input && nfi >= 2) f |= RF_SENS;
        if (type >= PDF_AND && type <= PDF_NOR) nfold = nfi - 1;
    }
    return type | (po ? 1u : 0u) << 4 | (nfi & 0xFFu) << 8 | f | nfold << 24;
}

PDF_HD uint32_t flagmask(uint32_t h, uint32_t f) { return (h & f) ? 0xFFFFFFFFu : 0u; }

// Gate evaluation on bit-planes, tracking the values under both vectors
// (V = vector 2, v1 = vector 1).  The reference folds the 2-input table left
// over the fan-ins (simkernel.cuh:142-148); every table is an exact
// per-vector function, so one step is AND with optional input/output
// inversion (De Morgan for OR/NOR).  NOT inverts both vectors.
PDF_HD void eval_first(uint32_t h, uint32_t fV, uint32_t fT, uint32_t &V, uint32_t &v1) {
    const uint32_t n = flagmask(h, RF_NOT);
    V = fV ^ n;
    v1 = fV ^ fT ^ n;
}
// FIX: the true n-input semantics, where a fold step may also be XOR and the
// result is inverted once at the end (RF_OINV) instead of per step.
template <bool FIX = false>
PDF_HD void eval_fold(uint32_t h, uint32_t &V, uint32_t &v1, uint32_t rV, uint32_t rT) {
    const uint32_t im = flagmask(h, RF_IM), x = im ^ flagmask(h, RF_OM);
    if (FIX) {
        const uint32_t xm = flagmask(h, RF_XOR);
        V = (xm & (V ^ rV)) | (~xm & (((V ^ im) & (rV ^ im)) ^ x));
        v1 = (xm & (v1 ^ rV ^ rT)) | (~xm & (((v1 ^ im) & (rV ^ rT ^ im)) ^ x));
    } else {
        V = ((V ^ im) & (rV ^ im)) ^ x;
        v1 = ((v1 ^ im) & (rV ^ rT ^ im)) ^ x;
    }
}
template <bool FIX = false>
PDF_HD void eval_finish(uint32_t h, uint32_t &V, uint32_t v1, uint32_t &T) {
    const uint32_t keep = ~flagmask(h, RF_KILL);
    T = (V ^ v1) & keep;
    V &= keep;
    if (FIX) V ^= flagmask(h, RF_OINV);  // inverting both vectors keeps the transition flag
}

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
// on 32 (on, off) code pairs at once.  ROBUST selects LUT_R, else LUT_NR.
//   AND/NAND LUT_NR 0x2A00: on=T0 & off in {S1,T1}  |  on=T1 & off=S1
//   AND/NAND LUT_R  0x2200: on in {T0,T1} & off=S1
//   OR/NOR   LUT_NR 0x5100: on=T0 & off=S0  |  on=T1 & off in {S0,T0}
//   OR/NOR   LUT_R  0x1100: on in {T0,T1} & off=S0
//   XOR/XNOR 0x0000: never
template <int ROBUST>
PDF_HD uint32_t sens_class(bool or_like, uint32_t onV, uint32_t onT, uint32_t offV, uint32_t offT) {
    if (or_like) return ROBUST ? (onT & ~offV & ~offT) : (onT & ~offV & (~offT | onV));
    return ROBUST ? (onT & offV & ~offT) : (onT & offV & (~onV | ~offT));
}
template <int ROBUST>
PDF_HD uint32_t sens(uint32_t type, uint32_t onV, uint32_t onT, uint32_t offV, uint32_t offT) {
    switch (type) {
        case PDF_AND:
        case PDF_NAND: return sens_class<ROBUST>(false, onV, onT, offV, offT);
        case PDF_OR:
        case PDF_NOR: return sens_class<ROBUST>(true, onV, onT, offV, offT);
        default: return 0;
    }
}

// The side-input test of a multi-input gate, OR over on-path candidates i
// of AND over side inputs x != i of sens(on = i, off = x)
// (markkernel.cuh:253-261 with robust()/nonrobust(), :43-72), in one pass
// over the fan-ins.  Every table above factors as
//   sens(i, x) = A1(i) & B1(x) | A2(i) & B2(x),   A1 & A2 = 0
//   AND/NAND LUT_R : A1 = T,        B1 = V & ~T     (A2 = 0)
//   OR/NOR   LUT_R : A1 = T,        B1 = ~V & ~T    (A2 = 0)
//   AND/NAND LUT_NR: A1 = T & ~V,   B1 = V;         A2 = T & V,  B2 = V & ~T
//   OR/NOR   LUT_NR: A1 = T & ~V,   B1 = ~V & ~T;   A2 = T & V,  B2 = ~V
// so AND_{x != i} sens(i, x) = A1(i) & E1(i) | A2(i) & E2(i) with
// Ek(i) = AND_{x != i} Bk(x) = Z0k | (Z1k & ~Bk(i)), where Z0k holds the
// pairs with no zero among all Bk(x) and Z1k those with exactly one.  The
// result is then Z0k & OR_i Ak(i) | Z1k & OR_i (Ak(i) & ~Bk(i)) over k.
struct SensAcc {
    uint32_t z0[2], z1[2], a[2], an[2];
};
PDF_HD void sens_init(SensAcc &s) {
    for (int k = 0; k < 2; k++) {
        s.z0[k] = 0xFFFFFFFFu;
        s.z1[k] = 0;
        s.a[k] = 0;
        s.an[k] = 0;
    }
}
PDF_HD void sens_term(SensAcc &s, int k, uint32_t A, uint32_t B) {
    const uint32_t n = ~B;
    s.z1[k] = (s.z1[k] & B) | (s.z0[k] & n);
    s.z0[k] &= B;
    s.a[k] |= A;
    s.an[k] |= A & n;
}
// Fan-in with value bit-planes (V, T).
template <int ROBUST>
PDF_HD void sens_step(SensAcc &s, bool or_like, uint32_t V, uint32_t T) {
    if (ROBUST) {
        sens_term(s, 0, T, (or_like ? ~V : V) & ~T);
    } else {
        sens_term(s, 0, T & ~V, or_like ? (~V & ~T) : V);
        sens_term(s, 1, T & V, or_like ? ~V : (V & ~T));
    }
}
template <int ROBUST>
PDF_HD uint32_t sens_result(const SensAcc &s) {
    uint32_t r = (s.z0[0] & s.a[0]) | (s.z1[0] & s.an[0]);
    if (!ROBUST) r |= (s.z0[1] & s.a[1]) | (s.z1[1] & s.an[1]);
    return r;
}

// The FIXED tables factor the same way, per gate class (and: AND/NAND, or:
// OR/NOR, xor: XOR/XNOR; masks all-ones for the gate's class, else zero):
//   robust     A1 = T & ~V (~V dropped for xor),  B1 = and: V,  or: ~V & ~T,  xor: ~T
//              A2 = T & V (none for xor),         B2 = and: V & ~T,  or: ~V
//   nonrobust  A1 = T,  B1 = and: V,  or: ~V,  xor: all
// and the candidate must carry a mark itself: Ak is ANDed with the fan-in's
// mark M, which makes the result OR_i (M(i) & AND_{x != i} sens(i, x)).
template <int NONROBUST>
PDF_HD void sens_step_fixed(SensAcc &s, uint32_t mand, uint32_t mor, uint32_t mxor, uint32_t V, uint32_t T,
                            uint32_t M) {
    if (NONROBUST) {
        sens_term(s, 0, T & M, (V & mand) | (~V & mor) | mxor);
    } else {
        sens_term(s, 0, T & M & (mxor | ~V), (V & mand) | (~V & ~T & mor) | (~T & mxor));
        sens_term(s, 1, T & V & M & ~mxor, (V & ~T & mand) | (~V & mor) | mxor);
    }
}

// A run of gates of one level, the unit of staging and of synchronisation.
struct __align__(16) Piece {
    uint32_t a, b;     // gates [a, b)
    uint32_t ea, eb;   // edge slice [ea, eb) to stage (16-byte aligned), or ea = eb = ~0: not staged
    uint32_t level;
    uint32_t far_off;  // its far fan-ins: far_ids[far_off .. far_off + far_n)
    uint32_t far_n;    // <= kMaxFar
    uint32_t nfar_n;   // far_n of the next piece, whose list starts at far_off + far_n rounded up to 4
};

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
