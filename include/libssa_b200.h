/*
 * libssa_b200.h -- extensions of the B200 libssa build beyond libssa.h.
 *
 * None of these has a counterpart in the reference API; the reference's own
 * entry points are declared, unchanged, in libssa.h.  They use the same global
 * settings (matrix, gap penalties, symbol type, chunk size, SIMD schedule) as
 * sw_align/nw_align and return the same alignment lists, freed with
 * free_alignment().
 */
#ifndef LIBSSA_B200_H_
#define LIBSSA_B200_H_

#include <stddef.h>
#include <stdint.h>

#include "libssa.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SSA_SMITH_WATERMAN 0
#define SSA_NEEDLEMAN_WUNSCH 1

/*
 * Batched search: every query of the batch is searched against the whole
 * database in shared device launches.  results[i] receives exactly the list
 * that sw_align/nw_align would return for queries[i] alone (same hits, same
 * tie order, same CIGARs).  Returns 0.  Errors follow the reference's
 * fatal() behaviour.
 */
int ssa_align_batch( int algorithm, p_query * queries, size_t n_queries, size_t hitcount, int bit_width,
        int align_type, p_alignment_list * results );

/* Counters of the last search call. */
typedef struct {
    uint64_t overflow_8_to_16;       /* sequences re-aligned at 16 bit */
    uint64_t overflow_16_to_64;      /* sequences re-aligned at 64 bit */
    uint64_t cells;                  /* sum over queries of query length x database residues */
    double gpu_seconds;              /* wall time of the last call's device pipeline, host replay included */
    uint64_t kernel_launches_total;  /* kernels launched by this process so far */
    double entry_seconds;            /* device time of the entry pass (all database pairs) */
    double kernel_seconds;           /* device time of entry pass, overflow passes and traceback */
    uint64_t h2d_bytes;              /* host-to-device bytes of the last call */
    uint64_t d2h_bytes;              /* device-to-host bytes of the last call */
} ssa_stats_t;

void ssa_get_stats( ssa_stats_t * out );

/* Measured packed-16x2 integer max throughput of the current device, in
 * lane operations per second (2 per instruction and thread), and the same as
 * warp instructions per clock per SM.  The denominator of the search kernels'
 * integer-pipe roofline.  Returns 0 on success. */
int ssa_b200_int_peak( double * lane_ops_per_second, double * instructions_per_clock_per_sm );

/* Marks the packed copy of the database stale, so the next search reads it
 * again through the plugin.  init_db() does this itself; call it after
 * loading a database into the plugin by other means. */
void ssa_db_refresh( void );

/* Number of residue codes of a query after mapping. */
size_t ssa_query_length( p_query p );

/*
 * Database plugin extension implemented by libsdb_b200 (the plugin that ships
 * with this build): installs count records from memory, record i being
 * residues[offsets[i] .. offsets[i+1]).  The data is copied.  Returns 0.
 */
int ssa_db_b200_load_memory( size_t count, const char * residues, const uint64_t * offsets );

#ifdef __cplusplus
}
#endif

#endif /* LIBSSA_B200_H_ */
