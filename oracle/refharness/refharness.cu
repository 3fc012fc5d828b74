// refharness.cu -- runs the reference's own kernels (unmodified, compiled by
// include path from the reference tree) on one case and dumps every result.
//
// TEST INFRASTRUCTURE ONLY: the output is a checker for the oracle
// (tests/golden/make_golden.py turns it into committed fixtures).
//
// The chunk loop below is ours; it calls the reference's four host functions
// in the order of main.cu:171-231 (segs = 1).
//
// Input file (little endian):
//   u32 G, u32 L, u32 n_pi, u32 robust, u64 n_vec, u64 chunk,
//   u32 level_offsets[L + 1], u8 type[G], u8 po[G], u32 nfi[G], u32 nfo[G],
//   u64 edge_offset[G], u64 n_edges, u32 edges[n_edges], u8 vec[n_pi][n_vec]
// Output file:
//   u64 n_chunks, u64 coverage[n_chunks], u8 sim[G][n_vec], u8 mark[G][n_vec],
//   i32 first_x[G], i32 first_y[G]
static int cover_flag = 0;
static int sim_flag = 0;
static int merge_flag = 0;
static int mark_flag = 0;
static int verbose_flag = 0;
static int robust_flag = 0;

#include "refshim.h"
#include "simkernel.cuh"
#include "markkernel.cuh"
#include "mergekernel.cuh"
#include "coverkernel.cuh"

namespace {

template <class T>
bool rd(FILE *f, T *p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }
template <class T>
void wr(FILE *f, const T *p, size_t n) { std::fwrite(p, sizeof(T), n, f); }

int fail(const char *m) {
    std::fprintf(stderr, "refharness: %s\n", m);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 3) return fail("usage: refharness <case.bin> <out.bin>");
    FILE *in = std::fopen(argv[1], "rb");
    if (!in) return fail("cannot open input");
    uint32_t G, L, n_pi, robust;
    uint64_t n_vec, chunk, n_edges;
    if (!rd(in, &G, 1) || !rd(in, &L, 1) || !rd(in, &n_pi, 1) || !rd(in, &robust, 1) || !rd(in, &n_vec, 1) ||
        !rd(in, &chunk, 1))
        return fail("short header");
    std::vector<uint32_t> lo(L + 1), nfi(G), nfo(G);
    std::vector<uint8_t> type(G), po(G), vec((size_t)n_pi * n_vec);
    std::vector<uint64_t> eo(G);
    if (!rd(in, lo.data(), L + 1) || !rd(in, type.data(), G) || !rd(in, po.data(), G) || !rd(in, nfi.data(), G) ||
        !rd(in, nfo.data(), G) || !rd(in, eo.data(), G) || !rd(in, &n_edges, 1))
        return fail("short netlist");
    std::vector<uint32_t> edges(n_edges);
    if (!rd(in, edges.data(), n_edges) || !rd(in, vec.data(), vec.size())) return fail("short body");
    std::fclose(in);
    robust_flag = robust ? 1 : 0;

    GPU_Circuit ckt;
    ckt.n = G;
    ckt.level_off = lo;
    ckt.nodes.resize(G);
    std::vector<GPUNODE> nodes(G);
    for (uint32_t g = 0; g < G; g++) {
        nodes[g] = GPUNODE{type[g], (int)nfi[g], (int)nfo[g], po[g], (uint32_t)eo[g]};
        ckt.nodes[g].typ = type[g];
    }
    if (cudaMalloc(&ckt.d_graph, sizeof(GPUNODE) * G) != cudaSuccess ||
        cudaMalloc(&ckt.d_offset, sizeof(uint32_t) * std::max<uint64_t>(n_edges, 1)) != cudaSuccess)
        return fail("cudaMalloc");
    cudaMemcpy(ckt.d_graph, nodes.data(), sizeof(GPUNODE) * G, cudaMemcpyHostToDevice);
    cudaMemcpy(ckt.d_offset, edges.data(), sizeof(uint32_t) * n_edges, cudaMemcpyHostToDevice);

    GPU_Data vecs(n_vec, n_pi, n_vec);
    cudaMemcpy2D(vecs.gpu(0).data, vecs.gpu(0).pitch, vec.data(), n_vec, n_vec, n_pi, cudaMemcpyHostToDevice);
    GPU_Data sim(n_vec, G, chunk);
    GPU_Data mark(n_vec, G, chunk);

    void *dc_segs = nullptr;
    int segments = 0;
    size_t startPattern = 0;
    std::vector<uint64_t> cov;
    for (unsigned int c = 0; c < sim.size(); c++) {  // main.cu:171-231
        uint64_t coverage = 0;
        gpuRunSimulation(sim, vecs, ckt, c, startPattern, c + 1 == sim.size());
        gpuMarkPaths(mark, sim, ckt, c, startPattern);
        gpuMergeSegments<1>(mark, sim, ckt, c, startPattern, &dc_segs, segments);
        gpuCountPaths<1>(ckt, mark, dc_segs, segments, &coverage, c, startPattern);
        cov.push_back(coverage);
        startPattern += mark.block_width();
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("CUDA error");

    std::vector<uint8_t> hs((size_t)G * n_vec), hm((size_t)G * n_vec);
    size_t s0 = 0;
    for (size_t c = 0; c < sim.size(); c++) {
        const size_t w = sim.gpu(c).width;
        cudaMemcpy2D(hs.data() + s0, n_vec, sim.gpu(c).data, sim.gpu(c).pitch, w, G, cudaMemcpyDeviceToHost);
        cudaMemcpy2D(hm.data() + s0, n_vec, mark.gpu(c).data, mark.gpu(c).pitch, w, G, cudaMemcpyDeviceToHost);
        s0 += w;
    }
    std::vector<segment<1, int2>> segs(G);
    cudaMemcpy(segs.data(), dc_segs, sizeof(segment<1, int2>) * G, cudaMemcpyDeviceToHost);
    std::vector<int32_t> fx(G), fy(G);
    for (uint32_t g = 0; g < G; g++) {
        fx[g] = segs[g].pattern.x;
        fy[g] = segs[g].pattern.y;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("CUDA error");

    FILE *out = std::fopen(argv[2], "wb");
    if (!out) return fail("cannot open output");
    const uint64_t nc = cov.size();
    wr(out, &nc, 1);
    wr(out, cov.data(), nc);
    wr(out, hs.data(), hs.size());
    wr(out, hm.data(), hm.size());
    wr(out, fx.data(), G);
    wr(out, fy.data(), G);
    std::fclose(out);
    vecs.release();
    sim.release();
    mark.release();
    return 0;
}
