// Test driver for libdmolp_dropin.so: calls the reference's C++ entry points as the reference's callers
// do and prints what they return as JSON lines for tests/test_dropin.py.  The same source, linked against
// the reference's own objects instead (oracle/Makefile target dropin_driver_ref), prints what the reference
// returns for the same calls (built with DMOLP_DRIVER_REFERENCE: the three functions the reference declares
// but never defines -- freeChunkSubgraph, runBoundaryLPOnGPU_Safe, cleanupGPUResources,
// include/phase2/gpu_lp_boundary.h:67,85,105 -- are not called there).
//
//   dropin_driver <graph.txt> <k> <theta> <iters> [--host-only]
//
// --host-only exercises the entry points that do no device work (loader, degree maps, hubs, first seed,
// subgraph and chunk construction).
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "dropin_types.hpp"

// the reference's declarations (include/phase1/*.h*, include/phase2/*.h)
void load_graph(const char *filename, int procId, int nprocs, std::unordered_map<int, std::vector<int>> &adj,
                std::unordered_map<int, int> &local_adj, int &V, uint64_t &E);
void gather_degrees(std::unordered_map<int, int> &local_degree, std::unordered_map<int, int> &global_degree,
                    int procId, int npros);
std::vector<int> find_hub_nodes(const std::unordered_map<int, int> &global_degree);
std::pair<int, int> find_first_seed(const std::unordered_map<int, int> &global_degree);
std::vector<int> find_seeds(const int procId, const int nprocs, const int numParts, const size_t num_nodes,
                            const std::pair<int, int> &first_seed, const std::vector<int> &hub_nodes,
                            const std::unordered_map<int, int> &global_degree,
                            const std::unordered_map<int, std::vector<int>> &adj);
void partition_expansion(int procId, int nprocs, int numParts, int theta, const std::vector<int> &seeds,
                         const std::unordered_map<int, int> &global_degree,
                         const std::unordered_map<int, std::vector<int>> &local_adj, Graph &local_partition_graphs,
                         GhostNodes &local_partition_ghosts, bool verbose);
void random_partition(int procId, int nprocs, int numParts, int theta, const std::vector<int> &seeds,
                      const std::unordered_map<int, int> &global_degree,
                      const std::unordered_map<int, std::vector<int>> &local_adj, Graph &local_partition_graphs,
                      GhostNodes &local_partition_ghosts, bool verbose);
Phase1Metrics run_phase1(int mpi_rank, int mpi_size, const char *graph_file, int num_parts, int theta, bool mode,
                         bool verbose, Graph &local_graph, GhostNodes &ghost_nodes);
PartitioningMetrics run_phase2(int mpi_rank, int mpi_size, int num_partitions, Graph &local_graph,
                               GhostNodes &ghost_nodes, int gpu_id);
BoundarySubgraph createBoundarySubgraphUnified(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                               const std::vector<int> &boundary_nodes,
                                               const std::vector<int> &local_labels,
                                               const std::vector<int> &ghost_labels, const std::vector<int> &global_ids,
                                               int num_local_nodes);
std::vector<int> expandBoundaryNodes(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                     const std::vector<int> &prev_boundary_nodes, const std::vector<int> &labels,
                                     const std::vector<double> &penalty, const std::vector<double> &RE,
                                     int labels_count, int iter);
GPULabelUpdateResult runBoundaryLPOnGPU_SubgraphUnified(const BoundarySubgraph &subgraph,
                                                        const std::vector<double> &penalty, int num_partitions);
GPULabelUpdateResult runBoundaryLPOnGPU_Chunked(const BoundarySubgraph &subgraph, const std::vector<double> &penalty,
                                                int num_partitions, size_t available_memory);
BoundarySubgraph createChunkSubgraph(const BoundarySubgraph &original, int start_node, int end_node);
void freeChunkSubgraph(BoundarySubgraph &chunk);
GPULabelUpdateResult runBoundaryLPOnGPU_Streaming(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                                                  const std::vector<int> &boundary_nodes,
                                                  const std::vector<int> &local_labels,
                                                  const std::vector<int> &ghost_labels,
                                                  const std::vector<int> &global_ids,
                                                  const std::vector<double> &penalty, int num_local_nodes,
                                                  int num_partitions, size_t max_memory_mb);
void runBoundaryLPOnGPU_Safe(const std::vector<int> &row_ptr, const std::vector<int> &col_idx,
                             const std::vector<int> &labels_old, std::vector<int> &labels_new,
                             const std::vector<double> &penalty, const std::vector<int> &boundary_nodes,
                             int num_partitions);
void cleanupGPUResources();

static std::string ivec(const std::vector<int> &v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + std::to_string(v[i]);
    return s + "]";
}

static uint64_t fnv(const std::vector<int> &v) {
    uint64_t h = 1469598103934665603ULL;
    const unsigned char *p = (const unsigned char *)v.data();
    for (size_t i = 0; i < v.size() * sizeof(int); ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

int main(int argc, char **argv) {
    if (argc < 5) return 2;
    const char *path = argv[1];
    const int k = atoi(argv[2]), theta = atoi(argv[3]), iters = atoi(argv[4]);
    const bool host_only = argc > 5 && strcmp(argv[5], "--host-only") == 0;

    std::unordered_map<int, std::vector<int>> adj;
    std::unordered_map<int, int> ldeg, gdeg;
    int V = 0;
    uint64_t E = 0;
    load_graph(path, 0, 1, adj, ldeg, V, E);
    gather_degrees(ldeg, gdeg, 0, 1);
    std::vector<int> hubs = find_hub_nodes(gdeg);
    std::pair<int, int> first = find_first_seed(gdeg);
    printf("{\"what\":\"host\",\"V\":%d,\"E\":%llu,\"hubs_hash\":\"%016llx\",\"num_hubs\":%zu,\"first\":[%d,%d]}\n", V,
           (unsigned long long)E, (unsigned long long)fnv(hubs), hubs.size(), first.first, first.second);

    // a subgraph of the first 20 vertices with modulo labels, and its chunks
    Graph rg;
    GhostNodes rgh;
    random_partition(0, 1, k, theta, {}, gdeg, adj, rg, rgh, false);
    std::vector<int> window;
    for (int v = 0; v < V && v < 20; ++v) window.push_back(v);
    BoundarySubgraph sg = createBoundarySubgraphUnified(rg.row_ptr, rg.col_indices, window, rg.vertex_labels, {},
                                                        rg.global_ids, rg.num_vertices);
    BoundarySubgraph ch = createChunkSubgraph(sg, 0, sg.num_nodes / 2);
    printf("{\"what\":\"subgraph\",\"nodes\":%d,\"edges\":%d,\"boundary\":%zu,\"mapping_hash\":\"%016llx\","
           "\"chunk_nodes\":%d,\"chunk_edges\":%d,\"random_labels_hash\":\"%016llx\",\"random_edges\":%d,"
           "\"random_row_ptr_hash\":\"%016llx\",\"random_col_hash\":\"%016llx\",\"random_vertices\":%d}\n",
           sg.num_nodes, sg.num_edges, sg.boundary_indices.size(), (unsigned long long)fnv(sg.node_mapping),
           ch.num_nodes, ch.num_edges, (unsigned long long)fnv(rg.vertex_labels), rg.num_edges,
           (unsigned long long)fnv(rg.row_ptr), (unsigned long long)fnv(rg.col_indices), rg.num_vertices);
#ifndef DMOLP_DRIVER_REFERENCE
    freeChunkSubgraph(ch);
#endif
    if (host_only) return 0;

    // lower-level phase 1 on the GPU
    std::vector<int> seeds = find_seeds(0, 1, k, V, first, hubs, gdeg, adj);
    Graph g1;
    GhostNodes gh1;
    partition_expansion(0, 1, k, theta, seeds, gdeg, adj, g1, gh1, false);
    printf("{\"what\":\"lower_phase1\",\"seeds\":%s,\"labels_hash\":\"%016llx\"}\n", ivec(seeds).c_str(),
           (unsigned long long)fnv(g1.vertex_labels));

    // run_phase1 + run_phase2 (iterations from DMOLP_LP_ITERATIONS, set by the test)
    Graph g;
    GhostNodes gh;
    Phase1Metrics m1 = run_phase1(0, 1, path, k, theta, false, false, g, gh);
    printf("{\"what\":\"phase1\",\"cut\":%d,\"vbal\":%.17g,\"ebal\":%.17g,\"vc\":%s,\"ec\":%s,\"labels_hash\":\"%016llx\","
           "\"E\":%llu}\n",
           m1.initial_edge_cut, m1.initial_vertex_balance, m1.initial_edge_balance,
           ivec(m1.partition_vertex_counts).c_str(), ivec(m1.partition_edge_counts).c_str(),
           (unsigned long long)fnv(g.vertex_labels), (unsigned long long)m1.total_edges);
    const std::vector<int> labels1 = g.vertex_labels;
    PartitioningMetrics m2 = run_phase2(0, 1, k, g, gh, 0);
    printf("{\"what\":\"phase2\",\"cut\":%d,\"vbal\":%.17g,\"ebal\":%.17g,\"labels_hash\":\"%016llx\",\"iters\":%d}\n",
           m2.edge_cut, m2.vertex_balance, m2.edge_balance, (unsigned long long)fnv(g.vertex_labels), iters);

    // one step through the single-step entry points from the phase-1 labels, with zero penalties
    std::vector<double> pen(k, 0.0), RE(k, 1.0);
    std::vector<int> all;
    for (int v = 0; v < V; ++v) all.push_back(v);
    std::vector<int> w = expandBoundaryNodes(g.row_ptr, g.col_indices, all, labels1, pen, RE, V, 1);
    GPULabelUpdateResult r1 = runBoundaryLPOnGPU_Streaming(g.row_ptr, g.col_indices, w, labels1, {}, g.global_ids,
                                                           pen, V, k, 512);
    BoundarySubgraph sub = createBoundarySubgraphUnified(g.row_ptr, g.col_indices, w, labels1, {}, g.global_ids, V);
    GPULabelUpdateResult r2 = runBoundaryLPOnGPU_SubgraphUnified(sub, pen, k);
    GPULabelUpdateResult r3 = runBoundaryLPOnGPU_Chunked(sub, pen, k, (size_t)1 << 40);
    int same4 = 1;
#ifndef DMOLP_DRIVER_REFERENCE
    std::vector<int> l4;
    runBoundaryLPOnGPU_Safe(g.row_ptr, g.col_indices, labels1, l4, pen, w, k);
    for (int i = 0; i < r1.change_count; ++i)
        if (l4[r1.updated_nodes[i]] != r1.updated_labels[i]) same4 = 0;
#endif
    // the window as a set (the reference returns it grouped by an unordered_map over labels, this library in
    // ascending ids; every consumer treats it as a set)
    std::vector<int> ws = w;
    std::sort(ws.begin(), ws.end());
    printf("{\"what\":\"single_step\",\"window\":%zu,\"window_set_hash\":\"%016llx\",\"changes\":[%d,%d,%d],"
           "\"same_nodes\":%d,\"safe_consistent\":%d}\n",
           ws.size(), (unsigned long long)fnv(ws), r1.change_count, r2.change_count, r3.change_count,
           (int)(r1.updated_nodes == r2.updated_nodes && r1.updated_labels == r2.updated_labels), same4);

    // the same step with penalties, through the chunked paths: the chunked entry point with room for one
    // chunk of the minimum size (1024 subgraph nodes) and the streaming entry point with no room at all
    std::vector<double> pen2(k);
    for (int p = 0; p < k; ++p) pen2[p] = 0.05 * (double)((p * 7) % 5 - 2);
    auto step_line = [&](const char *what, const GPULabelUpdateResult &r) {
        printf("{\"what\":\"%s\",\"changes\":%d,\"nodes_hash\":\"%016llx\",\"labels_hash\":\"%016llx\"}\n", what,
               r.change_count, (unsigned long long)fnv(r.updated_nodes), (unsigned long long)fnv(r.updated_labels));
    };
    step_line("step_unified", runBoundaryLPOnGPU_SubgraphUnified(sub, pen2, k));
    step_line("step_chunked", runBoundaryLPOnGPU_Chunked(sub, pen2, k, 1));
    step_line("step_streaming_chunked",
              runBoundaryLPOnGPU_Streaming(g.row_ptr, g.col_indices, w, labels1, {}, g.global_ids, pen2, V, k, 0));
    step_line("step_streaming",
              runBoundaryLPOnGPU_Streaming(g.row_ptr, g.col_indices, w, labels1, {}, g.global_ids, pen2, V, k, 512));
    printf("{\"what\":\"chunks\",\"subgraph_nodes\":%d,\"subgraph_edges\":%d}\n", sub.num_nodes, sub.num_edges);

    // -m random: random_partition's graph and labels, then phase 2 from them
    Graph gr;
    GhostNodes ghr;
    Phase1Metrics mr = run_phase1(0, 1, path, k, theta, true, false, gr, ghr);
    printf("{\"what\":\"random_phase1\",\"cut\":%d,\"E\":%d,\"row_ptr_hash\":\"%016llx\",\"col_hash\":\"%016llx\","
           "\"labels_hash\":\"%016llx\",\"vc\":%s}\n",
           mr.initial_edge_cut, gr.num_edges, (unsigned long long)fnv(gr.row_ptr), (unsigned long long)fnv(gr.col_indices),
           (unsigned long long)fnv(gr.vertex_labels), ivec(mr.partition_vertex_counts).c_str());
    PartitioningMetrics mr2 = run_phase2(0, 1, k, gr, ghr, 0);
    printf("{\"what\":\"random_phase2\",\"cut\":%d,\"vbal\":%.17g,\"ebal\":%.17g,\"labels_hash\":\"%016llx\"}\n",
           mr2.edge_cut, mr2.vertex_balance, mr2.edge_balance, (unsigned long long)fnv(gr.vertex_labels));
#ifndef DMOLP_DRIVER_REFERENCE
    cleanupGPUResources();
#endif
    return 0;
}
