// ORACLE / TEST INFRASTRUCTURE ONLY.  Compile-time check that the drop-in library's declarations of the
// reference's public types (dmolp_b200/csrc/dropin_types.hpp) have the reference's layout
// (include/graph_types.h, include/phase2/gpu_lp_boundary.h), so objects cross the boundary unchanged.
#include <cstddef>
#include <cstdint>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace mine {
#include "dropin_types.hpp"
}
#include "graph_types.h"
#include "phase2/gpu_lp_boundary.h"

#define SAME_SIZE(T) static_assert(sizeof(mine::T) == sizeof(::T), #T " size")
#define SAME_FIELD(T, f) static_assert(offsetof(mine::T, f) == offsetof(::T, f), #T "::" #f " offset")

SAME_SIZE(Graph);
SAME_FIELD(Graph, num_vertices);
SAME_FIELD(Graph, num_edges);
SAME_FIELD(Graph, row_ptr);
SAME_FIELD(Graph, col_indices);
SAME_FIELD(Graph, global_ids);
SAME_FIELD(Graph, vertex_labels);
SAME_SIZE(GhostNodes);
SAME_FIELD(GhostNodes, global_ids);
SAME_FIELD(GhostNodes, ghost_labels);
SAME_FIELD(GhostNodes, global_to_local);
SAME_SIZE(PartitionStats);
SAME_FIELD(PartitionStats, total_vertices);
SAME_FIELD(PartitionStats, total_edges);
SAME_FIELD(PartitionStats, expected_edges);
SAME_SIZE(Phase1Metrics);
SAME_FIELD(Phase1Metrics, initial_edge_cut);
SAME_FIELD(Phase1Metrics, initial_vertex_balance);
SAME_FIELD(Phase1Metrics, initial_edge_balance);
SAME_FIELD(Phase1Metrics, loading_time_ms);
SAME_FIELD(Phase1Metrics, distribution_time_ms);
SAME_FIELD(Phase1Metrics, total_vertices);
SAME_FIELD(Phase1Metrics, total_edges);
SAME_FIELD(Phase1Metrics, partition_vertex_counts);
SAME_FIELD(Phase1Metrics, partition_edge_counts);
SAME_SIZE(PartitioningMetrics);
SAME_FIELD(PartitioningMetrics, edge_cut);
SAME_FIELD(PartitioningMetrics, vertex_balance);
SAME_FIELD(PartitioningMetrics, edge_balance);
SAME_FIELD(PartitioningMetrics, loading_time_ms);
SAME_FIELD(PartitioningMetrics, distribution_time_ms);
SAME_FIELD(PartitioningMetrics, num_partitions);
SAME_FIELD(PartitioningMetrics, total_vertices);
SAME_FIELD(PartitioningMetrics, total_edges);
SAME_SIZE(BoundarySubgraph);
SAME_FIELD(BoundarySubgraph, row_ptr);
SAME_FIELD(BoundarySubgraph, boundary_indices);
SAME_FIELD(BoundarySubgraph, labels);
SAME_FIELD(BoundarySubgraph, num_nodes);
SAME_FIELD(BoundarySubgraph, num_edges);
SAME_FIELD(BoundarySubgraph, num_local_nodes);
SAME_SIZE(GPULabelUpdateResult);
SAME_FIELD(GPULabelUpdateResult, updated_nodes);
SAME_FIELD(GPULabelUpdateResult, updated_labels);
SAME_FIELD(GPULabelUpdateResult, change_count);
SAME_SIZE(Delta);

int main() { return 0; }
