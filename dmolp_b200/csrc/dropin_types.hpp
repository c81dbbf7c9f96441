// The data types of the reference's public C++ interface, declared here so the drop-in library builds
// without the reference tree.  Member order and types are those of include/graph_types.h:47-346 and
// include/phase2/gpu_lp_boundary.h:7-30 of the reference, so objects cross the boundary unchanged and the
// mangled names of the functions in dropin.cpp equal the reference's.  (Checked by a compile-time layout
// test against the reference headers where they are available.)  Printing helpers are not repeated.
#pragma once

#include <cstdint>
#include <unordered_map>
#include <unordered_set>
#include <vector>

struct Delta {
    int gid;
    int new_label;
};

struct Graph {
    int num_vertices = 0;
    int num_edges = 0;
    std::vector<int> row_ptr;
    std::vector<int> col_indices;
    std::vector<int> global_ids;
    std::vector<int> vertex_labels;
    void clear() {
        num_vertices = 0;
        num_edges = 0;
        row_ptr.clear();
        col_indices.clear();
        global_ids.clear();
        vertex_labels.clear();
    }
};

struct GhostNodes {
    std::vector<int> global_ids;
    std::vector<int> ghost_labels;
    std::unordered_map<int, int> global_to_local;
    void clear() {
        global_ids.clear();
        ghost_labels.clear();
        global_to_local.clear();
    }
};

struct PartitionStats {
    std::vector<int> local_vertex_counts;
    std::vector<int> local_edge_counts;
    std::vector<int> global_vertex_counts;
    std::vector<int> global_edge_counts;
    int total_vertices;
    uint64_t total_edges;
    double expected_vertices;
    double expected_edges;
};

struct Phase1Metrics {
    int initial_edge_cut = 0;
    double initial_vertex_balance = 0.0;
    double initial_edge_balance = 0.0;
    long loading_time_ms = 0;
    long distribution_time_ms = 0;
    int total_vertices = 0;
    uint64_t total_edges = 0;
    std::vector<int> partition_vertex_counts;
    std::vector<int> partition_edge_counts;
};

struct PartitioningMetrics {
    int edge_cut = 0;
    double vertex_balance = 0.0;
    double edge_balance = 0.0;
    long loading_time_ms = 0;
    long distribution_time_ms = 0;
    int num_partitions = 0;
    int total_vertices = 0;
    uint64_t total_edges = 0;
};

struct BoundarySubgraph {
    std::vector<int> row_ptr;
    std::vector<int> col_idx;
    std::vector<int> node_mapping;
    std::vector<int> reverse_mapping;
    std::vector<int> boundary_indices;
    std::vector<int> local_node_flags;
    std::vector<int> labels;
    int num_nodes;
    int num_edges;
    int num_local_nodes;
    BoundarySubgraph() : num_nodes(0), num_edges(0), num_local_nodes(0) {}
};

struct GPULabelUpdateResult {
    std::vector<int> updated_nodes;
    std::vector<int> updated_labels;
    int change_count;
    GPULabelUpdateResult() : change_count(0) {}
};
