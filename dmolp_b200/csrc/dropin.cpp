// libdmolp_dropin.so: the reference's C++ entry points (include/phase1/*.h*, include/phase2/*.h of DMOLP)
// with their exact signatures, implemented over the C-ABI of libdmolp_b200.so.  Linking the reference's
// main.cpp and utils.cpp against this library instead of its src/phase1 and src/phase2 objects runs the
// partitioning path on the B200 kernels.
//
// Scope: one process, one GPU (mpi_size must be 1; there are then no ghost vertices).  The device is the
// caller's current one when a context is first needed (the reference's allocateGPU sets it before phase 2),
// read through the shared CUDA runtime.
// Environment knobs (not in the reference): DMOLP_LP_ITERATIONS=N runs exactly N LP iterations instead of
// the reference's stopping rules; DMOLP_LP_LABEL_CAP=full scores every label < k instead of min(k,32).
//
// Where the reference calls MPI_Abort / exit(1) (unreadable graph file, an invalid label or an odd cut-arc
// count in phase 2) this library prints a message and exits with the same code; other failures throw
// std::runtime_error.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime_api.h>

#include "dmolp_b200.h"
#include "dropin_types.hpp"

namespace {

using Clock = std::chrono::high_resolution_clock;

long ms_since(Clock::time_point t) {
    return (long)std::chrono::duration_cast<std::chrono::milliseconds>(Clock::now() - t).count();
}

void check(int rc, const char *what) {
    if (rc != DMOLP_OK) throw std::runtime_error(std::string(what) + ": " + dmolp_last_error());
}

// The caller's current device, read through the shared CUDA runtime its own code (allocateGPU) uses.
int caller_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        d = 0;
    }
    return d;
}

void require_single_rank(int mpi_size, const char *fn) {
    if (mpi_size != 1)
        throw std::runtime_error(std::string(fn) + ": this library runs one process on one GPU (mpi_size must be 1)");
}

// A context with a resident graph, remembered by the identity of the host arrays it was uploaded from.
struct Resident {
    dmolp_ctx *ctx = nullptr;
    const void *rp = nullptr, *ci = nullptr;
    size_t nrp = 0, nci = 0;
    int64_t nv = 0;

    void ensure_ctx() {
        if (!ctx) check(dmolp_create(caller_device(), &ctx), "dmolp_create");
    }
    void upload(const std::vector<int64_t> &off, const std::vector<int> &col, const std::vector<int> *raw) {
        ensure_ctx();
        check(dmolp_graph_upload(ctx, (int64_t)off.size() - 1, (int64_t)col.size(), off.data(), col.data(),
                                 raw ? raw->data() : nullptr),
              "dmolp_graph_upload");
        nv = (int64_t)off.size() - 1;
        rp = ci = nullptr;
    }
    // Upload an int32 CSR unless it is the one already resident.
    void ensure_graph(const std::vector<int> &row_ptr, const std::vector<int> &col_idx) {
        ensure_ctx();
        if (rp == row_ptr.data() && nrp == row_ptr.size() && ci == col_idx.data() && nci == col_idx.size()) return;
        std::vector<int64_t> off(row_ptr.begin(), row_ptr.end());
        if (off.empty()) off.push_back(0);
        upload(off, col_idx, nullptr);
        remember(row_ptr, col_idx);
    }
    void remember(const std::vector<int> &row_ptr, const std::vector<int> &col_idx) {
        rp = row_ptr.data();
        nrp = row_ptr.size();
        ci = col_idx.data();
        nci = col_idx.size();
    }
    void destroy() {
        if (ctx) dmolp_destroy(ctx);
        ctx = nullptr;
        rp = ci = nullptr;
    }
};

Resident g_main;  // the partitioned graph
Resident g_sub;   // subgraphs handed to runBoundaryLPOnGPU_SubgraphUnified
std::mutex g_mu;

// sort_unique of each adjacency row (src/phase1/partition.cpp:50-53, 232); self-loops kept unless asked.
void csr_from_adj(const std::unordered_map<int, std::vector<int>> &adj, int64_t nv, bool drop_self_loops,
                  std::vector<int64_t> &off, std::vector<int> &col) {
    off.assign(nv + 1, 0);
    std::vector<std::vector<int>> rows(nv);
    for (const auto &kv : adj) {
        if (kv.first < 0 || kv.first >= nv) continue;
        std::vector<int> r = kv.second;
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        if (drop_self_loops) r.erase(std::remove(r.begin(), r.end(), kv.first), r.end());
        for (int x : r)
            if (x < 0 || x >= nv) throw std::runtime_error("neighbour id outside [0, V)");
        rows[kv.first] = std::move(r);
    }
    for (int64_t v = 0; v < nv; ++v) off[v + 1] = off[v] + (int64_t)rows[v].size();
    col.resize(off[nv]);
    for (int64_t v = 0; v < nv; ++v) std::copy(rows[v].begin(), rows[v].end(), col.begin() + off[v]);
}

void fill_graph(Graph &g, int64_t nv, const std::vector<int64_t> &off, const std::vector<int> &col,
                const std::vector<int> &labels) {
    if (off[nv] > 0x7fffffff) throw std::runtime_error("graph has 2^31 or more arcs: beyond Graph's int32 CSR");
    g.clear();
    g.num_vertices = (int)nv;
    g.num_edges = (int)off[nv];
    g.row_ptr.assign(off.begin(), off.end());
    g.col_indices = col;
    g.global_ids.resize(nv);
    std::iota(g.global_ids.begin(), g.global_ids.end(), 0);
    g.vertex_labels = labels;
}

std::vector<int> device_labels(Resident &r) {
    std::vector<int> lab(r.nv);
    check(dmolp_labels_get(r.ctx, lab.data()), "dmolp_labels_get");
    return lab;
}

// Reference tokenisation of one line (fast_atoi, src/phase1/init.cpp:15-23).
void parse_line(const char *p, const char *end, std::vector<int> &out) {
    while (p < end && *p) {
        int x = 0;
        while (p < end && (unsigned)(*p - '0') <= 9) x = x * 10 + (*p++ - '0');
        while (p < end && *p && (unsigned)(*p - '0') > 9) ++p;
        out.push_back(x);
    }
}

// find_hub_nodes' input is the degree map in its iteration order (src/phase1/init.cpp:139-177); the sort
// (std::sort's exact permutation) and the tangent rule run in the C-ABI library on all host threads.
std::vector<int> hubs_from_pairs(const std::vector<std::pair<int, int>> &sd) {
    const int64_t n = (int64_t)sd.size();
    std::vector<int32_t> ids(n), deg(n), hubs(n);
    for (int64_t i = 0; i < n; ++i) {
        ids[i] = sd[i].first;
        deg[i] = sd[i].second;
    }
    int64_t nh = 0;
    check(dmolp_find_hubs_pairs(n, ids.data(), deg.data(), hubs.data(), &nh), "dmolp_find_hubs_pairs");
    return std::vector<int>(hubs.begin(), hubs.begin() + nh);
}

void phase1_balance(const std::vector<int> &vc, const std::vector<int> &ec, int nv, int k, Phase1Metrics &m) {
    const double ev = (double)nv / k;  // phase1.cpp:141-153
    double mv = 0;
    for (int c : vc) mv = std::max(mv, c / ev);
    double tot = 0;
    for (int c : ec) tot += c;
    const double ee = tot / k;
    double me = 0;
    for (int c : ec) me = std::max(me, c / ee);
    m.initial_vertex_balance = mv;
    m.initial_edge_balance = me;
}

int lp_cap_from_env() {
    const char *s = std::getenv("DMOLP_LP_LABEL_CAP");
    return (s && std::strcmp(s, "full") == 0) ? DMOLP_LP_CAP_FULL : DMOLP_LP_CAP_REF;
}

// One synchronous LP update of `window` on the resident graph `r` with labels `labels`.
GPULabelUpdateResult lp_on(Resident &r, const std::vector<int> &labels, const std::vector<double> &penalty,
                           const std::vector<int> &window, int k) {
    check(dmolp_labels_set(r.ctx, labels.data()), "dmolp_labels_set");
    std::vector<int32_t> nodes(window.size() + 1), labs(window.size() + 1);
    int64_t n = 0;
    check(dmolp_lp_apply(r.ctx, k, lp_cap_from_env(), penalty.data(), window.data(), (int64_t)window.size(),
                         nodes.data(), labs.data(), &n),
          "dmolp_lp_apply");
    std::vector<std::pair<int, int>> ch;
    for (int64_t i = 0; i < n; ++i) ch.emplace_back(nodes[i], labs[i]);
    std::sort(ch.begin(), ch.end());
    GPULabelUpdateResult res;
    for (auto &c : ch) {
        res.updated_nodes.push_back(c.first);
        res.updated_labels.push_back(c.second);
    }
    res.change_count = (int)res.updated_nodes.size();
    return res;
}

}  // namespace

// ============================================================================ phase 1 (include/phase1)

// include/phase1/init.hpp:8 -- src/phase1/init.cpp:25-100 at one rank: adj[source] holds line source+1's
// tokens in file order (duplicates and self-loops included), inserted in ascending source order.
void load_graph(const char *filename, int procId, int nprocs, std::unordered_map<int, std::vector<int>> &adj,
                std::unordered_map<int, int> &local_degree, int &V, uint64_t &E) {
    require_single_rank(nprocs, "load_graph");
    (void)procId;
    FILE *fp = fopen(filename, "rb");
    if (!fp) {
        fprintf(stderr, "Process %d: Error opening file: %s\n", procId, filename);
        std::exit(1);
    }
    std::string data;
    {
        std::vector<char> buf(1 << 22);
        size_t n;
        while ((n = fread(buf.data(), 1, buf.size(), fp)) > 0) data.append(buf.data(), n);
        fclose(fp);
    }
    const size_t nl0 = data.find('\n');
    if (nl0 == std::string::npos) {
        fprintf(stderr, "[proc %d] Error opening file: %s\n", procId, filename);
        std::exit(1);
    }
    const int header_v = std::atoi(data.substr(0, std::min<size_t>(nl0, 63)).c_str());
    adj.reserve(header_v / nprocs * 2);
    local_degree.reserve(header_v / nprocs * 2);
    int source = 0;
    size_t start = nl0 + 1;
    while (true) {
        const size_t nl = data.find('\n', start);
        if (nl == std::string::npos) break;  // an unterminated last line is dropped
        auto &nbrs = adj[source];
        parse_line(data.data() + start, data.data() + nl, nbrs);
        ++source;
        start = nl + 1;
    }
    uint64_t e = 0;
    for (auto &kv : adj) {
        local_degree[kv.first] = (int)kv.second.size();
        e += (uint64_t)kv.second.size();
    }
    V = (int)adj.size();
    E = e / 2;
}

// include/phase1/init.hpp:9 -- src/phase1/init.cpp:102-137 at one rank (insertion in local_degree's order).
void gather_degrees(std::unordered_map<int, int> &local_degree, std::unordered_map<int, int> &global_degree,
                    int procId, int nprocs) {
    require_single_rank(nprocs, "gather_degrees");
    (void)procId;
    std::vector<std::pair<int, int>> send;
    send.reserve(local_degree.size());
    for (auto &kv : local_degree) send.emplace_back(kv.first, kv.second);
    global_degree.clear();
    global_degree.reserve(send.size());
    for (auto &p : send) global_degree[p.first] = p.second;
}

// include/phase1/init.hpp:10
std::vector<int> find_hub_nodes(const std::unordered_map<int, int> &global_degree) {
    return hubs_from_pairs(std::vector<std::pair<int, int>>(global_degree.begin(), global_degree.end()));
}

// include/phase1/init.hpp:11 -- including the reference's tie test, which compares a vertex id with the best
// degree (src/phase1/init.cpp:183).
std::pair<int, int> find_first_seed(const std::unordered_map<int, int> &global_degree) {
    std::pair<int, int> best(-1, -1);
    for (const auto &kv : global_degree)
        if (kv.second > best.second || (kv.second == best.second && kv.first < best.second)) best = kv;
    return best;
}

// include/phase1/seed.hpp:8 -- the radius-2 ball marking and hub scan run on the GPU.
std::vector<int> find_seeds(const int procId, const int nprocs, const int numParts, const size_t num_nodes,
                            const std::pair<int, int> &first_seed, const std::vector<int> &hub_nodes,
                            const std::unordered_map<int, int> &global_degree,
                            const std::unordered_map<int, std::vector<int>> &adj) {
    require_single_rank(nprocs, "find_seeds");
    std::vector<int> seeds = { first_seed.first };
    if (numParts <= 0 || hub_nodes.empty()) {
        if (procId == 0)
            std::cout << "Error: Invalid numParts (" << numParts << ") or empty hub_nodes" << std::endl;
        return seeds;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    const int64_t nv = (int64_t)num_nodes;
    std::vector<int64_t> off;
    std::vector<int> col, raw(nv, 0);
    csr_from_adj(adj, nv, false, off, col);
    for (const auto &kv : global_degree)
        if (kv.first >= 0 && kv.first < nv) raw[kv.first] = kv.second;
    g_main.upload(off, col, &raw);
    std::vector<int32_t> out(numParts);
    int32_t n = 0;
    check(dmolp_find_seeds(g_main.ctx, numParts, first_seed.first, hub_nodes.data(), (int64_t)hub_nodes.size(),
                           out.data(), &n),
          "dmolp_find_seeds");
    if (n < numParts && procId == 0)
        std::cout << "Warning: Could not find valid seed " << (n + 1) << " outside existing coverage" << std::endl;
    return std::vector<int>(out.begin(), out.begin() + n);
}

// include/phase1/partition.hpp:10 -- theta-limited growth on the GPU; the Graph is the reference's
// local CSR at one rank (rows sorted and de-duplicated, self-loops kept; no ghosts).  With fewer seeds
// than parts (undefined in the reference) the remaining parts start empty.
void partition_expansion(int procId, int nprocs, int numParts, int theta, const std::vector<int> &seeds,
                         const std::unordered_map<int, int> &global_degree,
                         const std::unordered_map<int, std::vector<int>> &local_adj, Graph &local_partition_graphs,
                         GhostNodes &local_partition_ghosts, bool verbose) {
    require_single_rank(nprocs, "partition_expansion");
    (void)procId;
    std::lock_guard<std::mutex> lk(g_mu);
    const int64_t nv = (int64_t)local_adj.size();
    std::vector<int64_t> off;
    std::vector<int> col, raw(nv, 0);
    csr_from_adj(local_adj, nv, false, off, col);
    for (const auto &kv : global_degree)
        if (kv.first >= 0 && kv.first < nv) raw[kv.first] = kv.second;
    g_main.upload(off, col, &raw);
    int32_t rounds = 0;
    check(dmolp_expand_partitions(g_main.ctx, numParts, theta, seeds.data(),
                                  (int32_t)std::min<size_t>(seeds.size(), (size_t)numParts), &rounds),
          "dmolp_expand_partitions");
    fill_graph(local_partition_graphs, nv, off, col, device_labels(g_main));
    local_partition_ghosts.clear();
    g_main.remember(local_partition_graphs.row_ptr, local_partition_graphs.col_indices);
    if (verbose)
        std::cout << "=== [Rank 0] CSR Summary ===\nVertices: " << nv << "\nEdges:    " << off[nv]
                  << "\nGhosts:   0\nRounds:   " << rounds << "\n";
}

// include/phase1/random.hpp:10 -- src/phase1/random.cpp:24-127 at one rank: label = id % k; rows sorted,
// de-duplicated and without self-loops.
void random_partition(int procId, int nprocs, int numParts, int theta, const std::vector<int> &seeds,
                      const std::unordered_map<int, int> &global_degree,
                      const std::unordered_map<int, std::vector<int>> &local_adj, Graph &local_partition_graphs,
                      GhostNodes &local_partition_ghosts, bool verbose) {
    require_single_rank(nprocs, "random_partition");
    (void)theta;
    (void)seeds;
    (void)global_degree;
    (void)verbose;
    const int64_t nv = (int64_t)local_adj.size();
    std::vector<int64_t> off;
    std::vector<int> col;
    csr_from_adj(local_adj, nv, true, off, col);
    std::vector<int> lab(nv);
    for (int64_t v = 0; v < nv; ++v) lab[v] = numParts > 0 ? (int)(v % numParts) : 0;
    fill_graph(local_partition_graphs, nv, off, col, lab);
    local_partition_ghosts.clear();
    std::cout << "[random_partition] Rank " << procId << " | locals=" << nv << " edges=" << off[nv] << " ghosts=0\n";
}

// include/phase1/phase1.h:7 -- src/phase1/phase1.cpp:18-161 at one rank.  mode = true is the modulo
// partition of random_partition.
Phase1Metrics run_phase1(int mpi_rank, int mpi_size, const char *graph_file, int num_parts, int theta, bool mode,
                         bool verbose, Graph &local_graph, GhostNodes &ghost_nodes) {
    require_single_rank(mpi_size, "run_phase1");
    std::lock_guard<std::mutex> lk(g_mu);
    Phase1Metrics m{};
    const auto t0 = Clock::now();
    // The text is parsed on the device into the resident graph (load_graph + the CSR build of
    // build_local_graph_and_ghosts); the caller's Graph gets a host copy of it.
    g_main.ensure_ctx();
    dmolp_ingest_info ii;
    if (dmolp_graph_load_adjtext(g_main.ctx, graph_file, &ii) != 0) {
        fprintf(stderr, "Process %d: Error opening file: %s (%s)\n", mpi_rank, graph_file, dmolp_last_error());
        std::exit(1);
    }
    const int64_t nv = ii.num_vertices, na = ii.num_arcs;
    std::vector<int64_t> off(nv + 1);
    std::vector<int> col(na);
    std::vector<int> raw(nv);
    check(dmolp_graph_get(g_main.ctx, off.data(), col.data(), raw.data()), "dmolp_graph_get");
    g_main.nv = nv;
    g_main.rp = g_main.ci = nullptr;
    const uint64_t e2 = (uint64_t)ii.num_tokens;
    m.loading_time_ms = ms_since(t0);
    const auto t1 = Clock::now();
    std::vector<int> lab;
    std::vector<int> vc(num_parts, 0), ec(num_parts, 0);
    if (mode) {  // random_partition: CSR without self-loops, label = id % k
        std::vector<int64_t> off2(nv + 1, 0);
        std::vector<int> col2;
        col2.reserve(col.size());
        for (int64_t v = 0; v < nv; ++v) {
            for (int64_t j = off[v]; j < off[v + 1]; ++j)
                if (col[j] != v) col2.push_back(col[j]);
            off2[v + 1] = (int64_t)col2.size();
        }
        off.swap(off2);
        col.swap(col2);
        lab.resize(nv);
        for (int64_t v = 0; v < nv; ++v) lab[v] = (int)(v % num_parts);
        g_main.upload(off, col, nullptr);
        check(dmolp_labels_set(g_main.ctx, lab.data()), "dmolp_labels_set");
        int64_t cut = 0;
        std::vector<int64_t> v64(num_parts), e64(num_parts);
        check(dmolp_metrics(g_main.ctx, num_parts, &cut, v64.data(), e64.data()), "dmolp_metrics");
        m.initial_edge_cut = (int)cut;
        for (int p = 0; p < num_parts; ++p) {
            vc[p] = (int)v64[p];
            ec[p] = (int)e64[p];
        }
    } else {  // the graph parsed above is already resident
        std::vector<int64_t> v64(num_parts), e64(num_parts);
        std::vector<int32_t> seeds(num_parts);
        dmolp_phase1_info info;
        check(dmolp_phase1(g_main.ctx, num_parts, theta, seeds.data(), v64.data(), e64.data(), &info),
              "dmolp_phase1");
        if (info.num_seeds_found < num_parts && mpi_rank == 0)
            std::cout << "Warning: Could not find valid seed " << (info.num_seeds_found + 1)
                      << " outside existing coverage (remaining seeds by seed completion)" << std::endl;
        lab = device_labels(g_main);
        m.initial_edge_cut = (int)info.initial_edge_cut;
        for (int p = 0; p < num_parts; ++p) {
            vc[p] = (int)v64[p];
            ec[p] = (int)e64[p];
        }
    }
    fill_graph(local_graph, nv, off, col, lab);
    ghost_nodes.clear();
    g_main.remember(local_graph.row_ptr, local_graph.col_indices);
    m.partition_vertex_counts = vc;
    m.partition_edge_counts = ec;
    phase1_balance(vc, ec, (int)nv, num_parts, m);
    m.distribution_time_ms = ms_since(t1);
    m.total_vertices = (int)nv;
    m.total_edges = e2 / 2;
    if (verbose) std::cout << "[dmolp-b200] phase 1 on GPU: V=" << nv << " arcs=" << off[nv] << "\n";
    return m;
}

// ============================================================================ phase 2 (include/phase2)

// include/phase2/phase2.h:7 -- src/phase2/phase2.cpp:256-449 at one rank, on the GPU.
PartitioningMetrics run_phase2(int mpi_rank, int mpi_size, int num_partitions, Graph &local_graph,
                               GhostNodes &ghost_nodes, int gpu_id) {
    require_single_rank(mpi_size, "run_phase2");
    if (!ghost_nodes.ghost_labels.empty()) throw std::runtime_error("run_phase2: ghost vertices need mpi_size > 1");
    std::lock_guard<std::mutex> lk(g_mu);
    const auto t0 = Clock::now();
    std::cout << "[Rank " << mpi_rank << "/" << mpi_size << "] Phase2 (B200, GPU " << gpu_id << ")" << std::endl;
    g_main.ensure_graph(local_graph.row_ptr, local_graph.col_indices);
    check(dmolp_labels_set(g_main.ctx, local_graph.vertex_labels.data()), "dmolp_labels_set");
    dmolp_lp_config cfg;
    cfg.mode = DMOLP_LP_MODE_REF;
    cfg.iterations = 0;
    cfg.cap = lp_cap_from_env();
    cfg.flags = 0;
    if (const char *it = std::getenv("DMOLP_LP_ITERATIONS")) {
        cfg.mode = DMOLP_LP_MODE_FIXED;
        cfg.iterations = std::atoi(it);
    }
    dmolp_lp_result r;
    const int rc = dmolp_lp_run(g_main.ctx, num_partitions, &cfg, &r, nullptr, 0);
    if (rc == DMOLP_ERR_BAD_LABELS) {  // phase2.cpp:239-250 aborts here
        printf("[EdgeCut] %s. Aborting.\n", dmolp_last_error());
        std::exit(2);
    }
    check(rc, "dmolp_lp_run");
    local_graph.vertex_labels = device_labels(g_main);
    PartitioningMetrics m2;
    m2.edge_cut = (int)r.edge_cut;
    m2.vertex_balance = r.vertex_balance;
    m2.edge_balance = r.edge_balance;
    m2.loading_time_ms = ms_since(t0);
    m2.distribution_time_ms = 0;
    m2.num_partitions = num_partitions;
    m2.total_vertices = (int)r.total_vertices;
    m2.total_edges = (uint64_t)r.total_edges;
    std::cout << "[Rank " << mpi_rank << "] Phase2 done: " << r.iterations_run << " iterations, edge-cut "
              << r.edge_cut << ", GPU " << r.gpu_ms << " ms" << std::endl;
    return m2;
}

// include/phase2/gpu_lp_boundary.h:33 -- gpu_lp_boundary.cu:26-178: window plus 1-hop neighbours,
// ascending original ids; CSR restricted to the subgraph; local flags; window positions of local vertices.
BoundarySubgraph createBoundarySubgraphUnified(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                               const std::vector<int> &boundary_nodes,
                                               const std::vector<int> &local_labels,
                                               const std::vector<int> &ghost_labels, const std::vector<int> &global_ids,
                                               int num_local_nodes) {
    (void)global_ids;
    BoundarySubgraph sg;
    sg.num_local_nodes = num_local_nodes;
    const int total = (int)(local_labels.size() + ghost_labels.size());
    const int rows = (int)row_ptr.size() - 1;
    std::vector<char> inc(total, 0);
    for (int b : boundary_nodes) {
        if (b < 0 || b >= total) continue;
        inc[b] = 1;
        if (b < rows)
            for (int e = row_ptr[b]; e < row_ptr[b + 1]; ++e)
                if (col_idx[e] >= 0 && col_idx[e] < total) inc[col_idx[e]] = 1;
    }
    for (int i = 0; i < total; ++i)
        if (inc[i]) sg.node_mapping.push_back(i);
    sg.num_nodes = (int)sg.node_mapping.size();
    sg.reverse_mapping.assign(total, -1);
    sg.labels.resize(sg.num_nodes);
    sg.local_node_flags.resize(sg.num_nodes);
    for (int i = 0; i < sg.num_nodes; ++i) {
        const int o = sg.node_mapping[i];
        sg.reverse_mapping[o] = i;
        if (o < num_local_nodes) {
            sg.labels[i] = local_labels[o];
            sg.local_node_flags[i] = 1;
        } else {
            const int gi = o - num_local_nodes;
            if (gi < 0 || gi >= (int)ghost_labels.size()) {
                printf("Warning: Invalid ghost node index %d for original node %d\n", gi, o);
                std::exit(1);
            }
            sg.labels[i] = ghost_labels[gi];
            sg.local_node_flags[i] = 0;
        }
    }
    sg.row_ptr.assign(sg.num_nodes + 1, 0);
    for (int i = 0; i < sg.num_nodes; ++i) {
        const int o = sg.node_mapping[i];
        if (o < rows)
            for (int e = row_ptr[o]; e < row_ptr[o + 1]; ++e) {
                const int n = col_idx[e];
                if (n >= 0 && n < total && sg.reverse_mapping[n] != -1) sg.col_idx.push_back(sg.reverse_mapping[n]);
            }
        sg.row_ptr[i + 1] = (int)sg.col_idx.size();
    }
    sg.num_edges = (int)sg.col_idx.size();
    for (int b : boundary_nodes)
        if (b >= 0 && b < num_local_nodes && sg.reverse_mapping[b] != -1)
            sg.boundary_indices.push_back(sg.reverse_mapping[b]);
    return sg;
}

// include/phase2/gpu_lp_boundary.h:43 -- on the GPU; the selected set comes back in ascending id order
// (the reference's order follows its per-label grouping; every consumer treats it as a set).
std::vector<int> expandBoundaryNodes(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                     const std::vector<int> &prev_boundary_nodes, const std::vector<int> &labels,
                                     const std::vector<double> &penalty, const std::vector<double> &RE,
                                     int labels_count, int iter) {
    (void)penalty;
    std::lock_guard<std::mutex> lk(g_mu);
    if (labels_count != (int)row_ptr.size() - 1)
        throw std::runtime_error("expandBoundaryNodes: ghost vertices need mpi_size > 1");
    g_main.ensure_graph(row_ptr, col_idx);
    check(dmolp_labels_set(g_main.ctx, labels.data()), "dmolp_labels_set");
    std::vector<int32_t> out(std::max<int64_t>(1, g_main.nv));
    int64_t n = 0;
    check(dmolp_window_select(g_main.ctx, (int)RE.size(), iter, RE.data(), prev_boundary_nodes.data(),
                              (int64_t)prev_boundary_nodes.size(), out.data(), &n),
          "dmolp_window_select");
    out.resize(n);
    return out;
}

// include/phase2/gpu_lp_boundary.h:54 -- the subgraph is uploaded to its own context.
GPULabelUpdateResult runBoundaryLPOnGPU_SubgraphUnified(const BoundarySubgraph &subgraph,
                                                        const std::vector<double> &penalty, int num_partitions) {
    std::lock_guard<std::mutex> lk(g_mu);
    std::vector<int64_t> off(subgraph.row_ptr.begin(), subgraph.row_ptr.end());
    if (off.empty()) off.push_back(0);
    g_sub.upload(off, subgraph.col_idx, nullptr);
    std::vector<int> window;
    for (int b : subgraph.boundary_indices)
        if (b >= 0 && b < subgraph.num_nodes && subgraph.local_node_flags[b] == 1) window.push_back(b);
    GPULabelUpdateResult sub = lp_on(g_sub, subgraph.labels, penalty, window, num_partitions);
    GPULabelUpdateResult res;
    for (int i = 0; i < sub.change_count; ++i) {
        res.updated_nodes.push_back(subgraph.node_mapping[sub.updated_nodes[i]]);
        res.updated_labels.push_back(sub.updated_labels[i]);
    }
    res.change_count = sub.change_count;
    return res;
}

// include/phase2/gpu_lp_boundary.h:67 -- gpu_lp_boundary.cu:633-675: rows [start,end) with only the arcs
// inside the chunk.
BoundarySubgraph createChunkSubgraph(const BoundarySubgraph &original, int start_node, int end_node) {
    BoundarySubgraph ch;
    const int n = end_node - start_node;
    if (n <= 0) return ch;
    ch.num_nodes = n;
    ch.labels.assign(original.labels.begin() + start_node, original.labels.begin() + end_node);
    ch.local_node_flags.assign(original.local_node_flags.begin() + start_node,
                               original.local_node_flags.begin() + end_node);
    ch.node_mapping.assign(original.node_mapping.begin() + start_node, original.node_mapping.begin() + end_node);
    for (int b : original.boundary_indices)
        if (b >= start_node && b < end_node) ch.boundary_indices.push_back(b - start_node);
    ch.row_ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (int j = original.row_ptr[start_node + i]; j < original.row_ptr[start_node + i + 1]; ++j) {
            const int nb = original.col_idx[j];
            if (nb >= start_node && nb < end_node) ch.col_idx.push_back(nb - start_node);
        }
        ch.row_ptr[i + 1] = (int)ch.col_idx.size();
    }
    ch.num_edges = (int)ch.col_idx.size();
    return ch;
}

// include/phase2/gpu_lp_boundary.h:68 (declared, never defined in the reference): release a chunk.
void freeChunkSubgraph(BoundarySubgraph &chunk) { chunk = BoundarySubgraph(); }

// include/phase2/gpu_lp_boundary.h:60 -- gpu_lp_boundary.cu:571-628: chunks of the subgraph in turn, each
// from the subgraph's original labels, cross-chunk arcs dropped.
GPULabelUpdateResult runBoundaryLPOnGPU_Chunked(const BoundarySubgraph &subgraph, const std::vector<double> &penalty,
                                                int num_partitions, size_t available_memory) {
    GPULabelUpdateResult total;
    std::vector<int> new_labels = subgraph.labels;
    const double avg = subgraph.num_nodes > 0 ? (double)subgraph.num_edges / subgraph.num_nodes : 0.0;
    const size_t per_node = (sizeof(int) * 5) + (size_t)(sizeof(int) * avg);
    const int max_nodes = std::max(1024, (int)(available_memory / (per_node + 1)));
    for (int s = 0; s < subgraph.num_nodes; s += max_nodes) {
        const int e = std::min(s + max_nodes, subgraph.num_nodes);
        BoundarySubgraph ch = createChunkSubgraph(subgraph, s, e);
        if (ch.num_nodes == 0 || ch.boundary_indices.empty()) continue;
        GPULabelUpdateResult r = runBoundaryLPOnGPU_SubgraphUnified(ch, penalty, num_partitions);
        for (size_t i = 0; i < r.updated_nodes.size(); ++i) {
            const int o = r.updated_nodes[i];
            if (o < (int)subgraph.reverse_mapping.size()) {
                const int si = subgraph.reverse_mapping[o];
                if (si != -1 && si >= s && si < e) new_labels[si] = r.updated_labels[i];
            }
        }
    }
    for (int i = 0; i < subgraph.num_nodes; ++i)
        if (subgraph.labels[i] != new_labels[i] && subgraph.local_node_flags[i] == 1) {
            total.updated_nodes.push_back(subgraph.node_mapping[i]);
            total.updated_labels.push_back(new_labels[i]);
            total.change_count++;
        }
    return total;
}

// include/phase2/gpu_lp_boundary.h:71 -- gpu_lp_boundary.cu:525-565.  Without ghosts the update runs on the
// resident graph (the subgraph of the reference holds every neighbour of the window, so the result is the
// same); with ghosts it goes through the reference's subgraph.  The B200's memory never needs chunking.
GPULabelUpdateResult runBoundaryLPOnGPU_Streaming(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                                  const std::vector<int> &boundary_nodes,
                                                  const std::vector<int> &local_labels,
                                                  const std::vector<int> &ghost_labels,
                                                  const std::vector<int> &global_ids,
                                                  const std::vector<double> &penalty, int num_local_nodes,
                                                  int num_partitions, size_t max_memory_mb) {
    // The reference sizes the subgraph against max_memory_mb and takes the chunked path when it does not fit
    // (gpu_lp_boundary.cu:541-563).  The subgraph's footprint is bounded by the whole graph's: when that bound
    // fits, so does the subgraph, and the resident path gives the same result; otherwise the subgraph is
    // built and measured exactly as the reference does.
    const size_t avail = max_memory_mb * 1024 * 1024;
    const size_t nodes_max = (size_t)num_local_nodes + ghost_labels.size();
    const size_t bound = (nodes_max + 1) * sizeof(int) + col_idx.size() * sizeof(int) + 2 * nodes_max * sizeof(int) +
                         nodes_max * sizeof(int) + boundary_nodes.size() * sizeof(int) + penalty.size() * sizeof(double);
    if (bound > avail) {
        BoundarySubgraph sg = createBoundarySubgraphUnified(row_ptr, col_idx, boundary_nodes, local_labels,
                                                            ghost_labels, global_ids, num_local_nodes);
        const size_t need = sg.row_ptr.size() * sizeof(int) + sg.col_idx.size() * sizeof(int) +
                            2 * sg.labels.size() * sizeof(int) + sg.local_node_flags.size() * sizeof(int) +
                            sg.boundary_indices.size() * sizeof(int) + penalty.size() * sizeof(double);
        if (need > avail) return runBoundaryLPOnGPU_Chunked(sg, penalty, num_partitions, avail);
        return runBoundaryLPOnGPU_SubgraphUnified(sg, penalty, num_partitions);
    }
    if (!ghost_labels.empty()) {
        BoundarySubgraph sg = createBoundarySubgraphUnified(row_ptr, col_idx, boundary_nodes, local_labels,
                                                            ghost_labels, global_ids, num_local_nodes);
        return runBoundaryLPOnGPU_SubgraphUnified(sg, penalty, num_partitions);
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_main.ensure_graph(row_ptr, col_idx);
    std::vector<int> window;
    for (int b : boundary_nodes)
        if (b >= 0 && b < num_local_nodes) window.push_back(b);
    return lp_on(g_main, local_labels, penalty, window, num_partitions);
}

// include/phase2/gpu_lp_boundary.h:85 (declared, never defined in the reference): labels_new = labels_old
// with the boundary nodes updated by one synchronous LP step.
void runBoundaryLPOnGPU_Safe(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                             const std::vector<int> &labels_old, std::vector<int> &labels_new,
                             const std::vector<double> &penalty, const std::vector<int> &boundary_nodes,
                             int num_partitions) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_main.ensure_graph(row_ptr, col_idx);
    std::vector<int> window;
    for (int b : boundary_nodes)
        if (b >= 0 && b < (int)row_ptr.size() - 1) window.push_back(b);
    GPULabelUpdateResult r = lp_on(g_main, labels_old, penalty, window, num_partitions);
    labels_new = labels_old;
    for (int i = 0; i < r.change_count; ++i) labels_new[r.updated_nodes[i]] = r.updated_labels[i];
}

// include/phase2/gpu_lp_boundary.h:95 (declared, never defined in the reference): same contract as _Safe.
void runBoundaryLPOnGPU_PinnedOptimized(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                        const std::vector<int> &labels_old, std::vector<int> &labels_new,
                                        const std::vector<double> &penalty, const std::vector<int> &boundary_nodes,
                                        int num_partitions) {
    runBoundaryLPOnGPU_Safe(row_ptr, col_idx, labels_old, labels_new, penalty, boundary_nodes, num_partitions);
}

// include/phase2/gpu_lp_boundary.h:104 (declared, never defined in the reference): free every device buffer.
void cleanupGPUResources() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_main.destroy();
    g_sub.destroy();
}
