// fcount.cpp -- command line with the reference's flags and output line
// (main.cu:24-235), on the C ABI of libpdf_b200.
//
//   fcount --bench CIRCUIT [--robust] [--fixed] [--segs 1] [--num_patterns N]
//          [--verbose [--sim] [--mark] [--merge] [--cover]] [--branches] [--device D]
//          VECTORS...
//
// For each vector file: one line on stdout,
//   <file>:<vectors>,<gates>,<segs>;<gpu ms>;<sim ms>;<mark ms>;<merge ms>;<cover ms>;<total>
// the layout of main.cu:233-234.  The total is the exact covered-path count
// (up to 2^128 - 1, decimal).  Times are milliseconds summed over the chunks.
// Without dumps the grading is the fused pdf_grade, timed on the device with
// CUDA events; its forward kernel (sim, mark, prune and merge in one launch)
// is reported in the sim field, with mark and merge 0.  With --verbose and a
// stage flag each chunk goes through the stage calls (pdf_sim,
// pdf_mark_forward, pdf_mark, pdf_merge, pdf_cover) as in main.cu:171-231,
// each timed on its own from the host (call to device idle), and
// the stage's planes are written to the reference's log files in the current
// directory: gpusim-p2.log (--sim), gpumark-full.log and gpumark.log
// (--mark), gpumerge.log (--merge; per segment with --segs N > 1).
#include <cuda_runtime.h>
#include <getopt.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "pdf.h"

namespace {

int verbose_flag = 0, sim_flag = 0, mark_flag = 0, merge_flag = 0, cover_flag = 0, robust_flag = 0,
    branches_flag = 0, fixed_flag = 0;

[[noreturn]] void die(const std::string &what) {
    std::cerr << "fcount: " << what << std::endl;
    std::exit(1);
}

void check(pdf_status st, const char *call) {
    if (st != PDF_OK) die(std::string(call) + ": " + pdf_status_string(st));
}

void check_cuda(cudaError_t e, const char *call) {
    if (e != cudaSuccess) die(std::string(call) + ": " + cudaGetErrorString(e));
}

std::string u128_string(uint64_t hi, uint64_t lo) {
    if (!hi) return std::to_string(lo);
    unsigned __int128 x = ((unsigned __int128)hi << 64) | lo;
    std::string s;
    while (x) {
        s.insert(s.begin(), char('0' + (int)(x % 10)));
        x /= 10;
    }
    return s;
}

void usage(const char *argv0) {
    std::printf("Usage: %s --bench CIRCUIT [options] VECTORS...\n", argv0);
    std::printf("\t--bench /path/to/ckt : the circuit; a name containing \"bench\" is read as ISCAS .bench,\n"
                "\t                       anything else as pdf-level text\n");
    std::printf("\t--segs N : Run fault grading over segments of length N, where 1 <= N <= 8\n");
    std::printf("\t--robust : robust sensitisation table (LUT_R) instead of the default (LUT_NR)\n");
    std::printf("\t--num_patterns N : vector pairs per pass (rounded up to a multiple of 32)\n");
    std::printf("\t--verbose with --sim / --mark / --merge / --cover : write gpusim-p2.log /\n"
                "\t                       gpumark-full.log and gpumark.log / gpumerge.log / gpucover.log\n");
    std::printf("\t--branches : .bench only, a FROM gate on every fan-out branch\n");
    std::printf("\t--fixed : true n-input gates and textbook side conditions (non-robust; robust\n"
                "\t          with --robust) instead of the reference's semantics\n");
    std::printf("\t--device N : CUDA device\n");
}

struct DevPlanes {
    uint32_t *p = nullptr;
    ~DevPlanes() {
        if (p) cudaFree(p);
    }
};

}  // namespace

int main(int argc, char *argv[]) {
    std::string infile;
    std::vector<std::string> benchmarks;
    int segs = 1, device = 0;
    uint64_t override_patterns = 0;
    static struct option long_options[] = {{"verbose", no_argument, &verbose_flag, 1},
                                           {"cover", no_argument, &cover_flag, 1},
                                           {"mark", no_argument, &mark_flag, 1},
                                           {"merge", no_argument, &merge_flag, 1},
                                           {"sim", no_argument, &sim_flag, 1},
                                           {"robust", no_argument, &robust_flag, 1},
                                           {"brief", no_argument, &verbose_flag, 0},
                                           {"branches", no_argument, &branches_flag, 1},
                                           {"fixed", no_argument, &fixed_flag, 1},
                                           {"help", no_argument, nullptr, 'h'},
                                           {"bench", required_argument, nullptr, 'b'},
                                           {"num_patterns", required_argument, nullptr, 'o'},
                                           {"segs", required_argument, nullptr, 's'},
                                           {"device", required_argument, nullptr, 'd'},
                                           {nullptr, 0, nullptr, 0}};
    while (true) {
        int option_index = 0;
        const int c = getopt_long(argc, argv, "b:s:o:d:h", long_options, &option_index);
        if (c == -1) break;
        switch (c) {
            case 0:
                break;
            case 'b':
                infile = optarg;
                break;
            case 'o':
                override_patterns = std::strtoull(optarg, nullptr, 10);
                if (!override_patterns) die("--num_patterns must be a positive integer");
                break;
            case 's':
                segs = std::atoi(optarg);
                if (segs < 1 || segs > 8) die("Segment lengths over 8 are not supported!");
                break;
            case 'd':
                device = std::atoi(optarg);
                break;
            case 'h':
                usage(argv[0]);
                return 0;
            default:
                usage(argv[0]);
                return 1;
        }
    }
    for (; optind < argc; optind++) benchmarks.emplace_back(argv[optind]);
    if (infile.empty()) die("--bench argument is required.");

    char msg[512] = {0};
    pdf_netbuf *nb = nullptr;
    if (infile.find("bench") != std::string::npos) {
        if (pdf_read_bench(infile.c_str(), branches_flag ? PDF_BENCH_BRANCHES : 0, &nb, msg, sizeof msg) != PDF_OK)
            die(msg);
    } else {
        std::clog << "presorted benchmark " << infile << " ";
        if (pdf_read_level(infile.c_str(), &nb, msg, sizeof msg) != PDF_OK) die(msg);
    }
    pdf_netlist nl;
    pdf_netbuf_view(nb, &nl);
    const uint32_t G = nl.n_gates, n_pi = nl.level_offsets[1];
    std::clog << "Circuit size is: " << G << "Levels: " << nl.n_levels << std::endl;

    pdf_circuit_opts co{};
    co.device = device;
    co.seg_len = (uint32_t)segs;
    co.mark_mode = fixed_flag ? (robust_flag ? PDF_MARK_FIXED_ROBUST : PDF_MARK_FIXED_NONROBUST)
                              : (robust_flag ? PDF_MARK_ROBUST : PDF_MARK_DEFAULT);
    pdf_circuit *ckt = nullptr;
    check(pdf_circuit_create(&nl, &co, &ckt), "pdf_circuit_create");
    pdf_circuit_info ci{};
    check(pdf_circuit_query(ckt, &ci), "pdf_circuit_query");
    const uint64_t n_first = ci.n_segments;  // first-detect entries: nets, or segments
    std::vector<uint32_t> seg_list;
    if (segs > 1) {
        std::clog << "Segments of " << segs << " nets: " << n_first << std::endl;
        seg_list.resize(n_first * segs);
        check(pdf_circuit_segments(ckt, seg_list.data()), "pdf_circuit_segments");
    }
    const bool dumps = verbose_flag && (sim_flag || mark_flag || merge_flag || cover_flag);

    for (const std::string &vector_file : benchmarks) {
        std::cerr << "Vector set " << vector_file << std::endl;
        uint64_t n_vec = 0;
        uint32_t width = 0;
        if (pdf_vectors_dim(vector_file.c_str(), &n_vec, &width) != PDF_OK) die("cannot read vectors from " + vector_file);
        std::cerr << "Vector size: " << n_vec << "x" << width << std::endl;
        if (width != n_pi)
            die(vector_file + ": vectors have " + std::to_string(width) + " bits, the circuit " +
                std::to_string(n_pi) + " inputs");
        std::vector<uint8_t> vec((size_t)n_pi * n_vec);
        check(pdf_vectors_read(vector_file.c_str(), n_pi, n_vec, vec.data()), "pdf_vectors_read");
        // pairs over the whole stream (the last pair wraps to vector 0), then chunked
        const uint64_t ld = (n_vec + 31) / 32;
        std::vector<uint32_t> hv(ld * n_pi), ht(ld * n_pi);
        check(pdf_pairs_from_vectors(vec.data(), n_pi, n_vec, ld, hv.data(), ht.data()), "pdf_pairs_from_vectors");
        uint64_t chunk = override_patterns ? override_patterns : std::min<uint64_t>(n_vec, 1u << 20);
        chunk = (chunk + 31) / 32 * 32;
        std::clog << "Maximum patterns per pass: " << chunk << " / " << n_vec << std::endl;

        pdf_state *st = nullptr;
        check(pdf_state_create(ckt, &st), "pdf_state_create");
        double gpu = 0, sim = 0, mark = 0, merge = 0, cover = 0;
        pdf_totals total{};
        if (!dumps) {
            check(pdf_state_profile(st, 1), "pdf_state_profile");
            for (uint64_t p0 = 0; p0 < n_vec; p0 += chunk) {
                const uint64_t n = std::min(chunk, n_vec - p0);
                pdf_pairs pr{hv.data() + p0 / 32, ht.data() + p0 / 32, n, ld, 0};
                pdf_totals batch{};
                check(pdf_grade(ckt, st, &pr, p0, nullptr, &batch, nullptr), "pdf_grade");
                check(pdf_state_snapshot(st, nullptr, nullptr, &total), "pdf_state_snapshot");
                std::cerr << "GPU Coverage: " << u128_string(batch.hi, batch.lo)
                          << ", total: " << u128_string(total.hi, total.lo) << std::endl;
            }
            double ms[3] = {0, 0, 0};
            uint32_t calls = 0;
            check(pdf_state_profile_read(st, ms, &calls), "pdf_state_profile_read");
            sim = ms[0];
            cover = ms[1];
            gpu = ms[2];
        } else {
            check_cuda(cudaSetDevice(device), "cudaSetDevice");
            const uint64_t cw = chunk / 32;
            DevPlanes dp, dv, dt, dm, dmf;
            check_cuda(cudaMalloc(&dp.p, 2 * n_pi * cw * 4), "cudaMalloc");
            check_cuda(cudaMalloc(&dv.p, (size_t)G * cw * 4), "cudaMalloc");
            check_cuda(cudaMalloc(&dt.p, (size_t)G * cw * 4), "cudaMalloc");
            check_cuda(cudaMalloc(&dm.p, (size_t)G * cw * 4), "cudaMalloc");
            check_cuda(cudaMalloc(&dmf.p, (size_t)G * cw * 4), "cudaMalloc");
            std::vector<uint32_t> hp((size_t)G * cw), hq((size_t)G * cw);
            std::vector<uint32_t> fx(n_first), fy(n_first);
            auto timed = [](auto fn) {
                const auto t0 = std::chrono::steady_clock::now();
                fn();
                check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
                return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            };
            for (uint64_t p0 = 0; p0 < n_vec; p0 += chunk) {
                const uint64_t n = std::min(chunk, n_vec - p0), w = (n + 31) / 32;
                const bool app = p0 != 0;
                check_cuda(cudaMemcpy2D(dp.p, cw * 4, hv.data() + p0 / 32, ld * 4, w * 4, n_pi, cudaMemcpyHostToDevice),
                           "cudaMemcpy2D");
                check_cuda(cudaMemcpy2D(dp.p + n_pi * cw, cw * 4, ht.data() + p0 / 32, ld * 4, w * 4, n_pi,
                                        cudaMemcpyHostToDevice),
                           "cudaMemcpy2D");
                pdf_pairs pr{dp.p, dp.p + n_pi * cw, n, cw, 1};
                const double t_sim = timed([&] { check(pdf_sim(ckt, &pr, dv.p, dt.p, cw, nullptr), "pdf_sim"); });
                double t_mark = 0;
                if (mark_flag) {
                    check(pdf_mark_forward(ckt, dv.p, dt.p, dmf.p, n, cw, nullptr), "pdf_mark_forward");
                    check_cuda(cudaMemcpy(hq.data(), dmf.p, (size_t)G * cw * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
                    check(pdf_dump_mark("gpumark-full.log", hq.data(), G, n, cw, p0, app), "pdf_dump_mark");
                }
                t_mark = timed([&] { check(pdf_mark(ckt, dv.p, dt.p, dm.p, n, cw, nullptr), "pdf_mark"); });
                const double t_merge =
                    timed([&] { check(pdf_merge(ckt, st, dv.p, dm.p, n, cw, p0, nullptr), "pdf_merge"); });
                pdf_totals batch{};
                const double t_cover = timed([&] {
                    if (cover_flag) {  // gpucover.log: the paths each input credits to each pair
                        std::vector<uint64_t> counts((size_t)n_pi * n * 2);
                        check(pdf_cover_counts(ckt, st, dm.p, n, cw, p0, counts.data(), &batch, nullptr),
                              "pdf_cover_counts");
                        check(pdf_dump_cover("gpucover.log", counts.data(), n_pi, n, p0, app), "pdf_dump_cover");
                    } else {
                        check(pdf_cover(ckt, st, dm.p, n, cw, p0, &batch, nullptr), "pdf_cover");
                    }
                });
                sim += t_sim;
                mark += t_mark;
                merge += t_merge;
                cover += t_cover;
                gpu += t_sim + t_mark + t_merge + t_cover;
                if (sim_flag) {
                    check_cuda(cudaMemcpy(hp.data(), dv.p, (size_t)G * cw * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
                    check_cuda(cudaMemcpy(hq.data(), dt.p, (size_t)G * cw * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
                    check(pdf_dump_sim("gpusim-p2.log", hp.data(), hq.data(), G, n, cw, p0, app), "pdf_dump_sim");
                }
                if (mark_flag) {
                    check_cuda(cudaMemcpy(hq.data(), dm.p, (size_t)G * cw * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
                    check(pdf_dump_mark("gpumark.log", hq.data(), G, n, cw, p0, app), "pdf_dump_mark");
                }
                check(pdf_state_snapshot(st, fx.data(), fy.data(), &total), "pdf_state_snapshot");
                if (merge_flag && segs > 1)
                    check(pdf_dump_segments("gpumerge.log", seg_list.data(), segs, n_first, fx.data(), fy.data()),
                          "pdf_dump_segments");
                else if (merge_flag)
                    check(pdf_dump_merge("gpumerge.log", fx.data(), fy.data(), G), "pdf_dump_merge");
                std::cerr << "GPU Coverage: " << u128_string(batch.hi, batch.lo)
                          << ", total: " << u128_string(total.hi, total.lo) << std::endl;
            }
        }
        if (total.flags & PDF_FLAG_OVERFLOW) std::cerr << "warning: the path count exceeded 2^128 - 1 (saturated)" << std::endl;
        std::cerr << "   GPU: " << gpu << " ms" << std::endl;
        std::cout << vector_file << ":" << n_vec << "," << G << "," << segs << ";" << gpu << ";" << sim << ";" << mark
                  << ";" << merge << ";" << cover << ";" << u128_string(total.hi, total.lo) << std::endl;
        pdf_state_destroy(st);
    }
    pdf_circuit_destroy(ckt);
    pdf_netbuf_free(nb);
    return 0;
}
