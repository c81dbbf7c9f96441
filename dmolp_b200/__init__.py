"""B200-native implementation of DMOLP's partitioning path (BFS/hub seeding + boundary label propagation)."""
