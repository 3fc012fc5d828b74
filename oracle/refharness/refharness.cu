// refharness.cu -- runs the reference's own kernels (unmodified, compiled by
// include path from the reference tree) on one case and dumps every result.
//
// TEST INFRASTRUCTURE ONLY: the output is a checker for the oracle
// (tests/golden/make_golden.py turns it into committed fixtures).
//
// The chunk loop below is ours; it calls the reference's four host functions
// in the order of main.cu:171-231, with segments of N = 1..4 nets
// (gpuMergeSegments<N>, gpuCountPaths<N>, main.cu:185-223).
//
// Input file (little endian):
//   u32 G, u32 L, u32 n_pi, u32 robust, u64 n_vec, u64 chunk,
//   u32 level_offsets[L + 1], u8 type[G], u8 po[G], u32 nfi[G], u32 nfo[G],
//   u64 edge_offset[G], u64 n_edges, u32 edges[n_edges], u8 vec[n_pi][n_vec],
//   then optionally u32 N, u64 S, u32 segments[S][N] (N > 1: the segment
//   list; absent or N <= 1: one segment per net)
// Output file:
//   u64 n_chunks, u64 coverage[n_chunks], u8 sim[G][n_vec], u8 mark[G][n_vec],
//   i32 first_x[S], i32 first_y[S]   (S = G for single nets)
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

// main.cu:171-231 for segments of N nets; the first pair ids per segment
// come back in fx, fy.
template <int N>
void run_chunks(GPU_Circuit &ckt, GPU_Data &vecs, GPU_Data &sim, GPU_Data &mark, void **dc_segs, int &segments,
                std::vector<uint64_t> &cov, std::vector<int32_t> &fx, std::vector<int32_t> &fy) {
    size_t startPattern = 0;
    for (unsigned int c = 0; c < sim.size(); c++) {
        uint64_t coverage = 0;
        gpuRunSimulation(sim, vecs, ckt, c, startPattern, c + 1 == sim.size());
        gpuMarkPaths(mark, sim, ckt, c, startPattern);
        gpuMergeSegments<N>(mark, sim, ckt, c, startPattern, dc_segs, segments);
        gpuCountPaths<N>(ckt, mark, *dc_segs, segments, &coverage, c, startPattern);
        cov.push_back(coverage);
        startPattern += mark.block_width();
    }
    std::vector<segment<N, int2>> segs(segments);
    cudaMemcpy(segs.data(), *dc_segs, sizeof(segment<N, int2>) * segments, cudaMemcpyDeviceToHost);
    fx.resize(segments);
    fy.resize(segments);
    for (int s = 0; s < segments; s++) {
        fx[s] = segs[s].pattern.x;
        fy[s] = segs[s].pattern.y;
    }
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
    uint32_t N = 1;
    uint64_t S = G;
    if (rd(in, &N, 1) && N > 1) {
        if (N > 4 || !rd(in, &S, 1)) return fail("bad segment header");
        std::vector<uint32_t> sg(S * N);
        if (!rd(in, sg.data(), sg.size())) return fail("short segment list");
        harness_segments().assign(sg.begin(), sg.end());
    } else {
        N = 1;
    }
    std::fclose(in);
    robust_flag = robust ? 1 : 0;
    // Shapes on which the reference's barriers never diverge: its merge kernel
    // syncs inside a test of the segment index (20 segments per block) and
    // of the pair index (128 pairs per warp row), mergekernel.cuh:130-173.
    if (S % 20 || chunk % 1024 || n_vec % 1024 || chunk > 4224)
        return fail("segments not a multiple of 20, or chunks not a multiple of 1,024 pairs up to 4,224");

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
    std::vector<uint64_t> cov;
    std::vector<int32_t> fx, fy;
    switch (N) {
        case 1: run_chunks<1>(ckt, vecs, sim, mark, &dc_segs, segments, cov, fx, fy); break;
        case 2: run_chunks<2>(ckt, vecs, sim, mark, &dc_segs, segments, cov, fx, fy); break;
        case 3: run_chunks<3>(ckt, vecs, sim, mark, &dc_segs, segments, cov, fx, fy); break;
        default: run_chunks<4>(ckt, vecs, sim, mark, &dc_segs, segments, cov, fx, fy); break;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("CUDA error");
    if (fx.size() != S) return fail("segment count differs from the list given");

    std::vector<uint8_t> hs((size_t)G * n_vec), hm((size_t)G * n_vec);
    size_t s0 = 0;
    for (size_t c = 0; c < sim.size(); c++) {
        const size_t w = sim.gpu(c).width;
        cudaMemcpy2D(hs.data() + s0, n_vec, sim.gpu(c).data, sim.gpu(c).pitch, w, G, cudaMemcpyDeviceToHost);
        cudaMemcpy2D(hm.data() + s0, n_vec, mark.gpu(c).data, mark.gpu(c).pitch, w, G, cudaMemcpyDeviceToHost);
        s0 += w;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("CUDA error");

    FILE *out = std::fopen(argv[2], "wb");
    if (!out) return fail("cannot open output");
    const uint64_t nc = cov.size();
    wr(out, &nc, 1);
    wr(out, cov.data(), nc);
    wr(out, hs.data(), hs.size());
    wr(out, hm.data(), hm.size());
    wr(out, fx.data(), fx.size());
    wr(out, fy.data(), fy.size());
    std::fclose(out);
    vecs.release();
    sim.release();
    mark.release();
    return 0;
}
