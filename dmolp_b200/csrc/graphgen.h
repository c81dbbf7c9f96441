// Seeded synthetic graph generators (host C++).  Outputs are undirected CSR graphs with sorted,
// de-duplicated neighbour lists, no self-loops, int64 offsets and int32 neighbour ids.
#ifndef DMOLP_GRAPHGEN_H
#define DMOLP_GRAPHGEN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dmolp_csr dmolp_csr;

const char *dmolp_gen_last_error(void);
int dmolp_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int permute,
                   dmolp_csr **out);
int dmolp_gen_knn(int64_t n, int dim, int knn, uint64_t seed, dmolp_csr **out);
int dmolp_gen_ba(int64_t n, int m, uint64_t seed, dmolp_csr **out);
/* Band graph: vertex i on a cycle of n with a reach w_i uniform in [wmin, wmax]; i ~ j when their distance on
 * the cycle is at most max(w_i, w_j).  Dense rows: with n = 65536, wmin = 12000, wmax = 24000 it has about
 * 2.6e9 arcs (beyond 32-bit arc offsets). */
int dmolp_gen_band(int64_t n, int wmin, int wmax, uint64_t seed, dmolp_csr **out);
int dmolp_csr_from_arrays(int64_t nv, int64_t narcs, const int64_t *off, const int32_t *col, dmolp_csr **out);
int64_t dmolp_csr_nv(const dmolp_csr *g);
int64_t dmolp_csr_narcs(const dmolp_csr *g);
int dmolp_csr_copy(const dmolp_csr *g, int64_t *off, int32_t *col);
int dmolp_csr_write_adjtext(const dmolp_csr *g, const char *path);
void dmolp_csr_free(dmolp_csr *g);
/* 64-bit FNV-1a over n bytes: the fingerprint the parity fixtures record for label arrays. */
uint64_t dmolp_fnv1a(const void *data, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
