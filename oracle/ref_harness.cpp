/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Drives the reference DMOLP sources, compiled unmodified
 * from where they lie (see oracle/Makefile), to produce golden outputs for the parity tests and
 * the timed CPU baseline.  Nothing in the product links or calls this.
 *
 * What it does:
 *   - phase 1: the reference's own run_phase1 (src/phase1/phase1.cpp:18), preceded by the same
 *     lower-level calls (load_graph, gather_degrees, find_hub_nodes, find_first_seed, find_seeds)
 *     so hubs/seeds can be dumped and so a seed list shorter than k (the reference then reads
 *     seeds[p] past the end, src/phase1/partition.cpp:347) is reported instead of executed.
 *   - phase 2, mode "ref": the reference's own run_phase2 (src/phase2/phase2.cpp:256).
 *   - phase 2, mode "fixed": the same per-iteration steps as phase2.cpp:295-416 for exactly N
 *     iterations (no early breaks; an empty window makes an iteration a no-op).
 *   In both modes the per-iteration LP call (runBoundaryLPOnGPU_Streaming,
 *   src/phase2/gpu_lp_boundary.cu:525) is routed through oracle_ref_streaming below, which either
 *   calls the reference's real GPU path (--gpu) or runs cpu_boundary_lp_kernel, a line-by-line CPU
 *   restatement of boundaryLPKernel_unified (gpu_lp_boundary.cu:327-427) over the reference's own
 *   subgraph (createBoundarySubgraphUnified, gpu_lp_boundary.cu:26).
 */
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

// Route run_phase2's LP call through the hook below (phase2.cpp:325).
#define runBoundaryLPOnGPU_Streaming oracle_ref_streaming
#include "phase2/phase2.cpp"
#undef runBoundaryLPOnGPU_Streaming

#include "phase1/init.hpp"
#include "phase1/seed.hpp"
#include "phase1/random.hpp"

// The reference's real implementation (gpu_lp_boundary.cu:525); the header above was read while the
// macro was active, so it is declared here under its own name.
GPULabelUpdateResult runBoundaryLPOnGPU_Streaming(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                                  const std::vector<int> &boundary_nodes,
                                                  const std::vector<int> &local_labels,
                                                  const std::vector<int> &ghost_labels,
                                                  const std::vector<int> &global_ids,
                                                  const std::vector<double> &penalty, int num_local_nodes,
                                                  int num_partitions, size_t max_memory_mb);

namespace {

bool g_use_gpu = false;
FILE *g_trace = nullptr;
int g_hook_calls = 0;

uint64_t fnv1a(const void *data, size_t n, uint64_t h = 1469598103934665603ULL) {
    const unsigned char *p = (const unsigned char *)data;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// Hash of a vertex SET (order-independent): sort a copy, then FNV-1a.
uint64_t set_hash(std::vector<int> v) {
    std::sort(v.begin(), v.end());
    return fnv1a(v.data(), v.size() * sizeof(int));
}

// Order-independent checksum of a vertex set: the sum (mod 2^64) of the SplitMix64 finaliser of each id.
// The CUDA path accumulates the same sum while it emits a window, so whole runs can be compared per
// iteration without copying windows back.
uint64_t set_sum(const std::vector<int> &v) {
    uint64_t s = 0;
    for (int x : v) {
        uint64_t z = (uint64_t)(uint32_t)x + 0x9e3779b97f4a7c15ULL;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        s += z ^ (z >> 31);
    }
    return s;
}

/*
 * CPU restatement of boundaryLPKernel_unified (gpu_lp_boundary.cu:327-427): one simulated warp per
 * boundary index; shared double histogram of neighbour labels < min(k,32) (:358-384); best starts at the
 * own label's RAW count or -1e300 (:388-390); per 32-label chunk, penalise positive scores (:397-403),
 * shuffle-down max with the left operand kept on ties (:407-414), strict > against best (:417-420).
 */
void cpu_boundary_lp_kernel(const BoundarySubgraph &sg, const std::vector<double> &penalty, int num_partitions,
                            std::vector<int> &labels_new) {
    const int WARP = 32;
    const int eff = std::min(num_partitions, 32);
    const int n = sg.num_nodes;
    const long nb = (long)sg.boundary_indices.size();
#pragma omp parallel for schedule(dynamic, 256)
    for (long w = 0; w < nb; ++w) {
        int v = sg.boundary_indices[w];
        if (v < 0 || v >= n) continue;
        if (sg.local_node_flags[v] != 1) continue;
        int my_label = sg.labels[v];
        double scores[32];  // the kernel's per-warp shared histogram
        for (int i = 0; i < 32; ++i) scores[i] = 0.0;
        for (int e = sg.row_ptr[v]; e < sg.row_ptr[v + 1]; ++e) {
            int u = sg.col_idx[e];
            if (u >= 0 && u < n) {
                int lu = sg.labels[u];
                if (lu >= 0 && lu < eff) scores[lu] += 1.0;
            }
        }
        int best_label = my_label;
        double best_score = (my_label >= 0 && my_label < eff) ? scores[my_label] : -1e300;
        for (int base = 0; base < eff; base += WARP) {
            double cs[32];
            int cl[32];
            for (int lane = 0; lane < WARP; ++lane) {
                cl[lane] = base + lane;
                cs[lane] = -1e300;
                if (cl[lane] < eff) {
                    double s = scores[cl[lane]];
                    if (s > 0.0) s *= (1.0 + penalty[cl[lane]]);
                    cs[lane] = s;
                }
            }
            for (int off = WARP / 2; off > 0; off >>= 1) {
                double ns[32];
                int nl[32];
                for (int lane = 0; lane < WARP; ++lane) {
                    int src = lane + off;
                    double os = src < WARP ? cs[src] : cs[lane];
                    int ol = src < WARP ? cl[src] : cl[lane];
                    ns[lane] = cs[lane];
                    nl[lane] = cl[lane];
                    if (os > cs[lane]) {
                        ns[lane] = os;
                        nl[lane] = ol;
                    }
                }
                std::memcpy(cs, ns, sizeof(cs));
                std::memcpy(cl, nl, sizeof(cl));
            }
            if (cs[0] > best_score) {
                best_score = cs[0];
                best_label = cl[0];
            }
        }
        labels_new[v] = best_label;
    }
}

void write_i32(const std::string &path, const std::vector<int> &v) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) {
        fprintf(stderr, "cannot write %s\n", path.c_str());
        exit(3);
    }
    if (!v.empty()) fwrite(v.data(), sizeof(int), v.size(), f);
    fclose(f);
}

std::vector<int> read_i32(const std::string &path) {
    std::vector<int> v;
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(3);
    }
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    v.resize(n / sizeof(int));
    if (n && fread(v.data(), sizeof(int), v.size(), f) != v.size()) exit(3);
    fclose(f);
    return v;
}

std::string json_ivec(const std::vector<int> &v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); ++i) {
        if (i) s += ",";
        s += std::to_string(v[i]);
    }
    return s + "]";
}

std::string json_dvec_bits(const std::vector<double> &v) {
    std::string s = "[";
    char buf[32];
    for (size_t i = 0; i < v.size(); ++i) {
        uint64_t b;
        std::memcpy(&b, &v[i], 8);
        snprintf(buf, sizeof(buf), "%s\"%016llx\"", i ? "," : "", (unsigned long long)b);
        s += buf;
    }
    return s + "]";
}

}  // namespace

// Per-iteration LP call used by run_phase2 (phase2.cpp:325) and by the fixed-iteration loop.
GPULabelUpdateResult oracle_ref_streaming(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                          const std::vector<int> &boundary_nodes,
                                          const std::vector<int> &local_labels,
                                          const std::vector<int> &ghost_labels, const std::vector<int> &global_ids,
                                          const std::vector<double> &penalty, int num_local_nodes,
                                          int num_partitions, size_t max_memory_mb) {
    ++g_hook_calls;
    if (g_trace) {
        fprintf(g_trace, "{\"hook\":%d,\"window\":%zu,\"window_hash\":\"%016llx\",\"penalty\":%s}\n", g_hook_calls,
                boundary_nodes.size(), (unsigned long long)set_hash(boundary_nodes),
                json_dvec_bits(penalty).c_str());
    }
    if (g_use_gpu)
        return runBoundaryLPOnGPU_Streaming(row_ptr, col_idx, boundary_nodes, local_labels, ghost_labels, global_ids,
                                            penalty, num_local_nodes, num_partitions, max_memory_mb);
    // Same steps as runBoundaryLPOnGPU_SubgraphUnified (gpu_lp_boundary.cu:440-520) with the kernel on the CPU.
    BoundarySubgraph sg = createBoundarySubgraphUnified(row_ptr, col_idx, boundary_nodes, local_labels,
                                                        ghost_labels, global_ids, num_local_nodes);
    std::vector<int> updated = sg.labels;
    cpu_boundary_lp_kernel(sg, penalty, num_partitions, updated);
    GPULabelUpdateResult r;
    for (int i = 0; i < sg.num_nodes; ++i) {
        if (sg.local_node_flags[i] == 1 && sg.labels[i] != updated[i]) {
            r.updated_nodes.push_back(sg.node_mapping[i]);
            r.updated_labels.push_back(updated[i]);
            r.change_count++;
        }
    }
    return r;
}

namespace {

struct Args {
    std::string graph, out, mode = "fixed", labels_in;
    int k = 0, theta = 0, iters = 20, threads = 1, repeat = 1;
    bool phase1_only = false, dump_seeds = true, load_only = false;
};

void usage() {
    fprintf(stderr,
            "ref_harness <graph.txt> <k> <theta> --out DIR [--mode ref|fixed] [--iters N] [--gpu]\n"
            "            [--threads T] [--phase1-only] [--labels-in FILE] [--no-seed-dump] [--repeat R]\n"
            "  --repeat R  (fixed mode) run phase 2 R times from the same start, one timing line each\n"
            "  --load-only time the reference's load_graph (src/phase1/init.cpp:25) on the file alone\n");
    exit(2);
}

// Fixed-iteration phase 2: the steps of phase2.cpp:295-416 for exactly `iters` iterations.
// Also counts traversed edges per iteration: deg over prev window, over candidates, over the selected
// window, plus one pass over all arcs for the statistics.  lp_seconds (and each trace record's "seconds",
// cumulative) times the reference's own steps only: penalties, window expansion, the LP step and applying
// its changes, the statistics and the edge cut; the traversed-edge count and the trace are not timed.
PartitioningMetrics run_phase2_fixed(int k, int iters, Graph &g, GhostNodes &gh, FILE *trace, double &lp_seconds,
                                     uint64_t &te_total) {
    using clk = std::chrono::high_resolution_clock;
    double busy = 0.0;
    auto since = [](clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); };
    auto t0 = clk::now();
    int prev_edge_cut = computeEdgeCut(g, g.vertex_labels, gh, 0);
    PartitionStats stats = computePartitionStats(g, g.vertex_labels, gh, k);
    std::vector<int> window;
    for (int i = 0; i < g.num_vertices; ++i) window.push_back(i);
    busy += since(t0);
    const int nv = g.num_vertices + (int)gh.ghost_labels.size();
    auto deg = [&](int v) -> uint64_t { return (uint64_t)(g.row_ptr[v + 1] - g.row_ptr[v]); };
    std::vector<char> mark(nv > 0 ? nv : 1, 0);
    std::vector<int> touched;
    te_total = 0;
    for (int iter = 0; iter < iters; ++iter) {
        auto ta = clk::now();
        auto pens = calculatePenalties(stats, k, iter + 1, 0);
        busy += since(ta);
        uint64_t te_prev = 0, te_cand = 0, te_sel = 0, te_stats = 0;
        // candidates = prev window plus its neighbours (gpu_lp_boundary.cu:207-240), for the TE count only
        touched.clear();
        auto touch = [&](int v) {
            if (v >= 0 && v < nv && !mark[v]) {
                mark[v] = 1;
                touched.push_back(v);
            }
        };
        for (int v : window) {
            if (v < 0 || v >= nv) continue;
            touch(v);
            if (v < g.num_vertices) {
                te_prev += deg(v);
                for (int e = g.row_ptr[v]; e < g.row_ptr[v + 1]; ++e) touch(g.col_indices[e]);
            }
        }
        for (int c : touched) {
            if (c < g.num_vertices) te_cand += deg(c);
            mark[c] = 0;
        }
        const size_t ncand = touched.size();
        ta = clk::now();
        window = expandBoundaryNodes(g.row_ptr, g.col_indices, window, g.vertex_labels, pens[0], pens[1], nv, iter + 1);
        int changes = 0;
        if (!window.empty()) {
            GPULabelUpdateResult r = oracle_ref_streaming(g.row_ptr, g.col_indices, window, g.vertex_labels,
                                                          gh.ghost_labels, g.global_ids, pens[0], g.num_vertices, k,
                                                          (size_t)1 << 20);
            for (int i = 0; i < r.change_count; ++i) g.vertex_labels[r.updated_nodes[i]] = r.updated_labels[i];
            changes = r.change_count;
            stats = computePartitionStats(g, g.vertex_labels, gh, k);
            prev_edge_cut = computeEdgeCut(g, g.vertex_labels, gh, 0);
            te_stats = (uint64_t)g.row_ptr[g.num_vertices];
        }
        busy += since(ta);
        for (int v : window) te_sel += deg(v);
        te_total += te_prev + te_cand + te_sel + te_stats;
        if (trace) {
            fprintf(trace,
                    "{\"iter\":%d,\"window\":%zu,\"window_hash\":\"%016llx\",\"window_sum\":\"%016llx\",\"candidates\":%zu,"
                    "\"changes\":%d,\"edge_cut\":%d,\"labels_hash\":\"%016llx\",\"vertex_counts\":%s,\"edge_counts\":%s,"
                    "\"penalty\":%s,\"RE\":%s,\"te\":[%llu,%llu,%llu,%llu],\"seconds\":%.6f}\n",
                    iter + 1, window.size(), (unsigned long long)set_hash(window), (unsigned long long)set_sum(window),
                    ncand, changes, prev_edge_cut,
                    (unsigned long long)fnv1a(g.vertex_labels.data(), g.vertex_labels.size() * sizeof(int)),
                    json_ivec(stats.global_vertex_counts).c_str(), json_ivec(stats.global_edge_counts).c_str(),
                    json_dvec_bits(pens[0]).c_str(), json_dvec_bits(pens[1]).c_str(), (unsigned long long)te_prev,
                    (unsigned long long)te_cand, (unsigned long long)te_sel, (unsigned long long)te_stats, busy);
            fflush(trace);
        }
    }
    lp_seconds = busy;
    // final metrics exactly as phase2.cpp:424-441
    PartitionStats fs = computePartitionStats(g, g.vertex_labels, gh, k);
    double max_v = 0.0, max_e = 0.0;
    for (int i = 0; i < k; ++i) {
        double rv = (fs.expected_vertices > 0) ? (double)fs.global_vertex_counts[i] / fs.expected_vertices : 1.0;
        double re = (fs.expected_edges > 0) ? (double)fs.global_edge_counts[i] / fs.expected_edges : 1.0;
        max_v = std::max(max_v, rv);
        max_e = std::max(max_e, re);
    }
    PartitioningMetrics m;
    m.edge_cut = prev_edge_cut;
    m.vertex_balance = max_v;
    m.edge_balance = max_e;
    m.num_partitions = k;
    m.total_vertices = fs.total_vertices;
    m.total_edges = fs.total_edges;
    return m;
}

std::string dbl_bits(double d) {
    uint64_t b;
    std::memcpy(&b, &d, 8);
    char buf[24];
    snprintf(buf, sizeof(buf), "\"%016llx\"", (unsigned long long)b);
    return buf;
}

}  // namespace

int main(int argc, char **argv) {
    Args a;
    std::vector<const char *> pos;
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        auto next = [&]() -> const char * {
            if (i + 1 >= argc) usage();
            return argv[++i];
        };
        if (s == "--out") a.out = next();
        else if (s == "--mode") a.mode = next();
        else if (s == "--iters") a.iters = atoi(next());
        else if (s == "--gpu") g_use_gpu = true;
        else if (s == "--threads") a.threads = atoi(next());
        else if (s == "--phase1-only") a.phase1_only = true;
        else if (s == "--labels-in") a.labels_in = next();
        else if (s == "--no-seed-dump") a.dump_seeds = false;
        else if (s == "--repeat") a.repeat = atoi(next());
        else if (s == "--load-only") a.load_only = true;
        else if (s.size() && s[0] == '-') usage();
        else pos.push_back(argv[i]);
    }
    if (pos.size() != 3 || a.out.empty()) usage();
    a.graph = pos[0];
    a.k = atoi(pos[1]);
    a.theta = atoi(pos[2]);
    if (a.mode != "ref" && a.mode != "fixed") usage();
    mkdir(a.out.c_str(), 0755);
    if (a.load_only) {
        // The reference's text loader alone: file -> adjacency map and local degrees, as run_phase1 calls it.
        omp_set_num_threads(a.threads > 0 ? a.threads : 1);
        int real_out = dup(1);
        if (!freopen((a.out + "/reference_stdout.log").c_str(), "w", stdout)) return 3;
        std::unordered_map<int, std::vector<int>> adj;
        std::unordered_map<int, int> ldeg;
        int V = 0;
        uint64_t E = 0;
        auto t0 = std::chrono::high_resolution_clock::now();
        load_graph(a.graph.c_str(), 0, 1, adj, ldeg, V, E);
        const double secs = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
        uint64_t tokens = 0;
        for (auto &kv : adj) tokens += kv.second.size();
        FILE *rs = fdopen(real_out, "w");
        fprintf(rs, "{\"load_seconds\":%.6f,\"V\":%d,\"E\":%llu,\"lines\":%zu,\"tokens\":%llu}\n", secs, V,
                (unsigned long long)E, adj.size(), (unsigned long long)tokens);
        fclose(rs);
        return 0;
    }
    omp_set_num_threads(a.threads > 0 ? a.threads : 1);

    // The reference prints a lot from inside its functions; keep our own stdout for the summary.
    int real_stdout = dup(1);
    if (!freopen((a.out + "/reference_stdout.log").c_str(), "w", stdout)) return 3;

    FILE *p1 = fopen((a.out + "/phase1.json").c_str(), "w");
    if (!p1) return 3;
    bool phase1_undefined = false;

    // Seed pre-check with the reference's own lower-level calls (phase1.cpp:44-60).
    {
        std::unordered_map<int, std::vector<int>> adj;
        std::unordered_map<int, int> ldeg, gdeg;
        int V;
        uint64_t E;
        load_graph(a.graph.c_str(), 0, 1, adj, ldeg, V, E);
        gather_degrees(ldeg, gdeg, 0, 1);
        std::vector<int> hubs = find_hub_nodes(gdeg);
        std::pair<int, int> first = find_first_seed(gdeg);
        std::vector<int> seeds = find_seeds(0, 1, a.k, V, first, hubs, gdeg, adj);
        fprintf(p1, "{\"V\":%d,\"E\":%llu,\"first_seed\":[%d,%d],\"num_hubs\":%zu,\"hubs\":%s,\"seeds\":%s", V,
                (unsigned long long)E, first.first, first.second, hubs.size(),
                a.dump_seeds ? json_ivec(hubs).c_str() : "null", json_ivec(seeds).c_str());
        if ((int)seeds.size() < a.k) {
            // partition_expansion would index seeds[p] past the end (partition.cpp:347): undefined.
            fprintf(p1, ",\"unpinned\":\"fewer than k seeds (%zu < %d)\"", seeds.size(), a.k);
            if (a.labels_in.empty()) {
                fprintf(p1, "}\n");
                fclose(p1);
                FILE *rs = fdopen(real_stdout, "w");
                fprintf(rs, "{\"unpinned\":\"fewer than k seeds\",\"seeds\":%zu}\n", seeds.size());
                return 0;
            }
            phase1_undefined = true;
        }
    }

    Graph g;
    GhostNodes gh;
    auto t_p1 = std::chrono::high_resolution_clock::now();
    Phase1Metrics m1;
    if (!phase1_undefined) {
        m1 = run_phase1(0, 1, a.graph.c_str(), a.k, a.theta, false, false, g, gh);
    } else {
        // Phase 2 from given labels only: build the Graph with the reference's random_partition
        // (src/phase1/random.cpp:24-127; same CSR as partition_expansion for graphs without self-loops).
        std::unordered_map<int, std::vector<int>> adj;
        std::unordered_map<int, int> ldeg, gdeg;
        int V;
        uint64_t E;
        load_graph(a.graph.c_str(), 0, 1, adj, ldeg, V, E);
        gather_degrees(ldeg, gdeg, 0, 1);
        std::vector<int> none;
        random_partition(0, 1, a.k, a.theta, none, gdeg, adj, g, gh, false);
    }
    double p1_seconds = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t_p1).count();
    fprintf(p1,
            ",\"initial_edge_cut\":%d,\"initial_vertex_balance\":%s,\"initial_edge_balance\":%s,"
            "\"partition_vertex_counts\":%s,\"partition_edge_counts\":%s,\"num_vertices\":%d,\"num_edges\":%d,"
            "\"ghosts\":%zu,\"seconds\":%.6f}\n",
            m1.initial_edge_cut, dbl_bits(m1.initial_vertex_balance).c_str(),
            dbl_bits(m1.initial_edge_balance).c_str(), json_ivec(m1.partition_vertex_counts).c_str(),
            json_ivec(m1.partition_edge_counts).c_str(), g.num_vertices, g.num_edges, gh.global_ids.size(),
            p1_seconds);
    fclose(p1);
    write_i32(a.out + "/labels1.bin", g.vertex_labels);
    write_i32(a.out + "/row_ptr.bin", g.row_ptr);
    write_i32(a.out + "/col_idx.bin", g.col_indices);

    FILE *rs = fdopen(real_stdout, "w");
    if (a.phase1_only) {
        fprintf(rs, "{\"phase1_seconds\":%.6f}\n", p1_seconds);
        return 0;
    }
    if (!a.labels_in.empty()) {
        std::vector<int> l = read_i32(a.labels_in);
        if ((int)l.size() != g.num_vertices) {
            fprintf(stderr, "labels-in size %zu != V %d\n", l.size(), g.num_vertices);
            return 3;
        }
        g.vertex_labels = l;
    }

    g_trace = fopen((a.out + "/trace.jsonl").c_str(), "w");
    double lp_seconds = 0.0;
    uint64_t te_total = 0;
    PartitioningMetrics m2;
    if (a.mode == "ref") {
        auto t0 = std::chrono::high_resolution_clock::now();
        m2 = run_phase2(0, 1, a.k, g, gh, 0);
        lp_seconds = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
    } else {
        FILE *tr = g_trace;
        g_trace = nullptr;  // the fixed loop writes richer per-iteration records itself
        const std::vector<int> start = g.vertex_labels;
        for (int rep = 0; rep < std::max(1, a.repeat); ++rep) {
            g.vertex_labels = start;
            m2 = run_phase2_fixed(a.k, a.iters, g, gh, rep == 0 ? tr : nullptr, lp_seconds, te_total);
            if (a.repeat > 1) {
                FILE *rs0 = fdopen(dup(real_stdout), "w");
                fprintf(rs0, "{\"repeat\":%d,\"lp_seconds\":%.6f,\"te_total\":%llu,\"edge_cut\":%d}\n", rep,
                        lp_seconds, (unsigned long long)te_total, m2.edge_cut);
                fclose(rs0);
            }
        }
        g_trace = tr;
    }
    if (g_trace) fclose(g_trace);
    write_i32(a.out + "/labels2.bin", g.vertex_labels);
    FILE *r = fopen((a.out + "/result.json").c_str(), "w");
    fprintf(r,
            "{\"mode\":\"%s\",\"iters\":%d,\"hook_calls\":%d,\"edge_cut\":%d,\"vertex_balance\":%s,"
            "\"edge_balance\":%s,\"total_vertices\":%d,\"total_edges\":%llu,\"lp_seconds\":%.6f,"
            "\"te_total\":%llu,\"threads\":%d,\"gpu\":%d}\n",
            a.mode.c_str(), a.iters, g_hook_calls, m2.edge_cut, dbl_bits(m2.vertex_balance).c_str(),
            dbl_bits(m2.edge_balance).c_str(), m2.total_vertices, (unsigned long long)m2.total_edges, lp_seconds,
            (unsigned long long)te_total, a.threads, g_use_gpu ? 1 : 0);
    fclose(r);
    fprintf(rs, "{\"edge_cut\":%d,\"lp_seconds\":%.6f,\"te_total\":%llu,\"hook_calls\":%d}\n", m2.edge_cut,
            lp_seconds, (unsigned long long)te_total, g_hook_calls);
    fflush(rs);
    return 0;
}
