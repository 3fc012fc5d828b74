// refshim.h -- stand-ins for the reference's missing `util` submodule.
//
// TEST INFRASTRUCTURE ONLY (oracle/refharness builds oracle/_ref/refharness,
// used as a checker).  The reference's kernels (simkernel.cuh, markkernel.cuh,
// mergekernel.cuh, coverkernel.cuh) include util/*.h from an empty git
// submodule.  This file supplies, in our own code, the minimum of those
// contracts that the kernels use, reconstructed from their call sites:
//   GPUNODE{type,nfi,nfo,offset,po} + FIN (simkernel.cuh:108-145,
//   markkernel.cuh:220-223,277), GPUCKT (simkernel.cuh:97,108), GPU_Circuit
//   (levels()/levelsize()/size()/gpu()/offset(), simkernel.cuh:213-214,
//   markkernel.cuh:334), GPU_Data chunks of pitched gate-major byte rows
//   (simkernel.cuh:109, main.cu:149,163), coalesce_t (4 pair bytes per word),
//   GPU_DATA_type + REF2D (row y, column x), segment<N,int2> with a
//   sentinel-terminated list (mergekernel.cuh:215), and the S0..T1 / gate codes.
// CUDA 12 removed texture references; `texture<T, d>` becomes a
// __constant__ table read with point sampling and clamping, which is what
// the reference's unnormalised tex2D/tex1D fetches of integer coordinates do.
#ifndef REFSHIM_H
#define REFSHIM_H

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

// Gate codes: AND..XNOR must be 2..7 (markkernel.cuh:49 indexes LUT[type-2]);
// the others only need to be distinct.  Same numbering as include/pdf.h.
#define UNKN 0
#define INPT 1
#define AND 2
#define NAND 3
#define OR 4
#define NOR 5
#define XOR 6
#define XNOR 7
#define BUFF 8
#define NOT 9
#define FROM 10
#define DFF 11

#define S0 0
#define S1 1
#define T0 2
#define T1 3

#define MAX_BLOCKS 65535
#define DPRINT(...) \
    do {            \
    } while (0)

union coalesce_t {
    uint32_t packed;
    uint8_t rows[4];
    __host__ __device__ coalesce_t() {}
    __host__ __device__ coalesce_t(uint32_t p) : packed(p) {}
    __host__ __device__ coalesce_t(uint8_t a, uint8_t b, uint8_t c, uint8_t d) {
        rows[0] = a;
        rows[1] = b;
        rows[2] = c;
        rows[3] = d;
    }
    __host__ __device__ operator uint32_t() const { return packed; }
};

template <class T>
struct GPU_DATA_type {
    T *data;
    size_t pitch, width, height;
};

template <class T>
struct ARRAY2D {
    T *data;
    size_t pitch, width, height;
};

// REF2D(array, x, y): column x (pattern word), row y (gate).
template <class T>
__host__ __device__ __forceinline__ T &REF2D(const GPU_DATA_type<T> &a, size_t x, size_t y) {
    return *((T *)((char *)a.data + y * a.pitch) + x);
}
template <class T>
__host__ __device__ __forceinline__ T &REF2D(T *data, size_t pitch, size_t x, size_t y) {
    return *((T *)((char *)data + y * pitch) + x);
}
template <class T>
__host__ __device__ __forceinline__ const T &REF2D(const T *data, size_t pitch, size_t x, size_t y) {
    return *((const T *)((const char *)data + y * pitch) + x);
}

#define FIN(AR, OFF, ID) ((AR)[(OFF) + (ID)])

struct GPUNODE {
    int type;
    int nfi;
    int nfo;
    int po;
    uint32_t offset;
};

struct GPUCKT {
    GPUNODE *graph;
    uint32_t *offset;
};

struct NODEINFO {
    int typ;
};

class Circuit {
   public:
    std::vector<NODEINFO> nodes;
    const NODEINFO &at(size_t i) const { return nodes[i]; }
};

class GPU_Circuit : public Circuit {
   public:
    GPUNODE *d_graph = nullptr;
    uint32_t *d_offset = nullptr;
    std::vector<uint32_t> level_off;  // n_levels + 1
    size_t n = 0;
    size_t size() const { return n; }
    uint32_t levels() const { return (uint32_t)level_off.size() - 2; }  // loops run i <= levels()
    int levelsize(uint32_t i) const { return (int)(level_off[i + 1] - level_off[i]); }
    GPUNODE *gpu() const { return d_graph; }
    uint32_t *offset() const { return d_offset; }
};

inline GPUCKT toPod(const GPU_Circuit &c) { return GPUCKT{c.d_graph, c.d_offset}; }

// Pitched device rows, split along the pattern axis into chunks.
class GPU_Data {
   public:
    std::vector<ARRAY2D<uint8_t>> chunks;
    size_t bw = 0, h = 0, total = 0;
    GPU_Data(size_t total_width, size_t height, size_t block_width) : bw(block_width), h(height), total(total_width) {
        for (size_t s = 0; s < total_width; s += block_width) {
            ARRAY2D<uint8_t> a{};
            a.width = std::min(block_width, total_width - s);
            a.height = height;
            if (cudaMallocPitch((void **)&a.data, &a.pitch, a.width, height) != cudaSuccess) {
                std::fprintf(stderr, "refshim: cudaMallocPitch failed\n");
                std::exit(2);
            }
            cudaMemset2D(a.data, a.pitch, 0, a.width, height);
            chunks.push_back(a);
        }
    }
    ARRAY2D<uint8_t> &gpu(size_t chunk = 0) { return chunks[chunk]; }
    size_t size() const { return chunks.size(); }
    size_t block_width() const { return bw; }
    size_t height() const { return h; }
    size_t width() const { return total; }
    void unload() {}
    void release() {
        for (auto &a : chunks) cudaFree(a.data);
        chunks.clear();
    }
};

template <class T>
GPU_DATA_type<T> toPod(GPU_Data &d, size_t chunk = 0) {
    ARRAY2D<uint8_t> &a = d.gpu(chunk);
    return GPU_DATA_type<T>{(T *)a.data, a.pitch, a.width, a.height};
}

template <int N, class T>
struct segment {
    struct {
        int num[N];
    } key;
    T pattern;
};

// The segment list the harness was given ([S][N] gate ids: the reference's
// generator lives in its missing util/segment.cuh, so the harness feeds the
// list of the build under test); empty: one segment per net.
inline std::vector<int> &harness_segments() {
    static std::vector<int> v;
    return v;
}

// The segment list, terminated by a sentinel whose key is not a gate
// (mergekernel.cuh:215): for N = 1 without a given list, one segment per
// net, indexed by gate id.
template <int N>
void generateSegmentList(segment<N, int2> **out, const GPU_Circuit &ckt) {
    const std::vector<int> &src = harness_segments();
    const size_t S = src.empty() ? (N == 1 ? ckt.size() : 0) : src.size() / N;
    segment<N, int2> *l = new segment<N, int2>[S + 1];
    for (size_t s = 0; s < S; s++) {
        for (int i = 0; i < N; i++) l[s].key.num[i] = src.empty() ? (int)s : src[s * N + i];
        l[s].pattern = make_int2(-1, -1);
    }
    for (int i = 0; i < N; i++) l[S].key.num[i] = -1;
    *out = l;
}

// Timing helpers (used for the reference's elapsed-ms return values).
inline timespec diff(timespec a, timespec b) {
    timespec r;
    r.tv_sec = b.tv_sec - a.tv_sec;
    r.tv_nsec = b.tv_nsec - a.tv_nsec;
    if (r.tv_nsec < 0) {
        r.tv_sec -= 1;
        r.tv_nsec += 1000000000L;
    }
    return r;
}
inline float floattime(timespec t) { return (float)(t.tv_sec * 1e3 + t.tv_nsec / 1e6); }
inline float elapsed(timespec start) {
    timespec now;
    clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &now);
    return floattime(diff(start, now));
}
inline void gpuCheckMemory() {}

// ---- texture references -> __constant__ tables ----
template <class T, int D>
struct ref_tex_t {
    int w, h;
    T data[16];
};

template <class T, int D>
__device__ __forceinline__ T tex2D(const ref_tex_t<T, D> &t, float x, float y) {
    int ix = (int)floorf(x), iy = (int)floorf(y);
    ix = ix < 0 ? 0 : (ix >= t.w ? t.w - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= t.h ? t.h - 1 : iy);
    return t.data[iy * t.w + ix];
}
template <class T, int D>
__device__ __forceinline__ T tex1D(const ref_tex_t<T, D> &t, float x) {
    int ix = (int)floorf(x);
    ix = ix < 0 ? 0 : (ix >= t.w ? t.w - 1 : ix);
    return t.data[ix];
}

// cudaBindTextureToArray: copy the cudaArray's contents into the table.
template <class T, int D>
cudaError_t ref_bind_texture(const ref_tex_t<T, D> &sym, cudaArray_t arr, cudaChannelFormatDesc) {
    cudaChannelFormatDesc d;
    cudaExtent ext;
    unsigned int flags;
    cudaError_t e = cudaArrayGetInfo(&d, &ext, &flags, arr);
    if (e != cudaSuccess) return e;
    ref_tex_t<T, D> host{};
    host.w = (int)ext.width;
    host.h = ext.height ? (int)ext.height : 1;
    if ((size_t)host.w * host.h > 16) return cudaErrorInvalidValue;
    e = cudaMemcpy2DFromArray(host.data, host.w * sizeof(T), arr, 0, 0, host.w * sizeof(T), host.h,
                              cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(sym, &host, sizeof host);
}

#define texture __constant__ ref_tex_t
#define cudaBindTextureToArray ref_bind_texture

#endif
