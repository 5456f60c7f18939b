/* Synthetic input generators for the GIR-B200 benchmarks and tests (host-only, OpenMP).
 *
 * These have no counterpart in the reference's library: the reference reads graphs from its
 * four-file CSR (gir_constructor/graph.cpp:2-120) or builds them in memory
 * (graph::fromEdges, gir_constructor/graph.cpp:123-136). gir_gen_csr produces exactly the
 * arrays that loader reads, and gir_write_four_files writes them in its on-disk layout.
 *
 * All calls return 0 on success; on failure a non-zero code and gir_gen_last_error() text.
 * Arrays returned through int32_t** / uint32_t** are malloc'd; release them with gir_gen_free.
 */
#ifndef GIR_GEN_H
#define GIR_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* gir_gen_last_error(void);
void gir_gen_free(void* p);
uint64_t gir_gen_hash3(uint64_t seed, uint64_t a, uint64_t b);

/* Directed R-MAT edge list (a, b, c; d = 1 - a - b - c). `scale` quadrant levels per draw,
 * ids >= V and self-loops rejected, duplicates dropped keeping the earliest draw. With
 * target_unique > 0 the generator keeps drawing until that many distinct edges exist and
 * returns exactly that many; otherwise it uses exactly n_draws draws. permute != 0 applies a
 * seeded random permutation to the vertex ids. */
int gir_gen_rmat(int scale, int64_t V, int64_t n_draws, int64_t target_unique, double a, double b, double c,
                 uint64_t seed, int permute, int64_t* n_out, int32_t** src_out, int32_t** dst_out);

/* side x side 4-neighbour lattice with remove_frac of its edges removed and
 * longrange_frac * (#lattice edges) Pareto(pareto_shape)-length long-range edges added, both
 * directions of every undirected edge, weight = round(100 * Euclidean length) + U[0,50]. */
int gir_gen_lattice(int64_t side, double remove_frac, double longrange_frac, double pareto_shape,
                    uint64_t seed, int64_t* n_out, int32_t** src_out, int32_t** dst_out, uint32_t** w_out);

/* Forward + backward CSR (int32 offsets, rows sorted) of an edge list; optional per-edge
 * weights w_in are returned in forward-CSR order in w_fw. fw_beg/bw_beg hold V+1 entries. */
int gir_gen_csr(int64_t V, int64_t n, const int32_t* src, const int32_t* dst, const uint32_t* w_in,
                int32_t* fw_beg, int32_t* fw_adj, int32_t* bw_beg, int32_t* bw_adj, uint32_t* w_fw);

/* w(u,v) = lo + hash(seed,u,v) mod (hi-lo+1) for every forward-CSR entry. */
void gir_gen_uniform_weights(int64_t V, const int32_t* fw_beg, const int32_t* fw_adj, uint32_t lo, uint32_t hi,
                             uint64_t seed, uint32_t* w_out);

/* n uniform source vertices in [0, V). */
void gir_gen_sources(int64_t V, int64_t n, uint64_t seed, int32_t* out);

/* A batch of n_ins uniform inserts and n_del deletions sampled from the CSR's edges, shuffled. */
void gir_gen_updates(int64_t V, const int32_t* fw_beg, const int32_t* fw_adj, int64_t n_ins, int64_t n_del,
                     uint64_t seed, int32_t* u_out, int32_t* v_out, uint8_t* ins_out);

/* Writes <dir>fw_begin.bin, fw_adjacent.bin, bw_begin.bin, bw_adjacent.bin (int32). `dir` is
 * used as a prefix, as the reference does: pass it with its trailing '/'. */
int gir_write_four_files(const char* dir, int64_t V, const int32_t* fw_beg, const int32_t* fw_adj,
                         const int32_t* bw_beg, const int32_t* bw_adj);

#ifdef __cplusplus
}
#endif

#endif /* GIR_GEN_H */
