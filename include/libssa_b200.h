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

/*
 * Long-pair batch: queries[i] is aligned against the database sequence with ID
 * db_ids[i] (0-based, in plugin order) and nothing else.  results[i] receives
 * exactly the list that sw_align/nw_align(queries[i], 1, bit_width,
 * align_type) returns against a database holding only that sequence: one hit
 * with its score (and CIGAR and coordinates for COMPUTE_ALIGNMENT), or an
 * empty list for an empty sequence; db_seq.ID is db_ids[i].  A reference
 * caller does this with one init_db and one sw_align/nw_align per pair
 * (src/libssa.c:126-132, :229-251).  One warp scores each pair exactly, which
 * is what every entry width of the reference reports for one sequence, as
 * long as the width holds the score table and gap costs untruncated.  Returns
 * 0; -1 (message on stderr) for settings outside that: a table entry or
 * gapO + gapE outside the width's range, positive gap costs, a translated or
 * two-strand setup, an ID past the database.  Other errors follow fatal().
 */
int ssa_align_pairs( int algorithm, p_query * queries, const size_t * db_ids, size_t n_pairs, int bit_width,
        int align_type, p_alignment_list * results );

/* Device memory (bytes) for the direction matrices of one traceback wave: the
 * hits of a call whose matrices do not fit together are traced back in
 * several waves.  0 (the default) = the free device memory less a reserve. */
void ssa_b200_set_traceback_memory( size_t bytes );

/* Device memory (bytes) for the packed database.  A database that needs more
 * is streamed: its sequences, in segments of the length order, take turns on
 * the device during each search (each segment's entry pass and overflow
 * cascade run while it is resident), and the hits' sequences are gathered for
 * the traceback; results are the same.  The server (ssa_server_start) needs a
 * resident database.  0 (the default) = 40% of the device memory.  Takes
 * effect at the next search. */
void ssa_b200_set_db_memory( size_t bytes );

/* 1 if the current database is streamed, else 0 (packs it first if needed). */
int ssa_b200_db_streamed( void );

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

/* The overflow counters of ssa_get_stats per query of the last search call
 * (sw_align/nw_align: one query; ssa_align_batch: queries[i] at index i), as
 * the reference reports them for each sw_align/nw_align call
 * (src/algo/manager.c:156-159).  Writes min(n, count) entries of each non-NULL
 * array and returns count, the number of queries of that call. */
size_t ssa_b200_query_overflows( uint64_t * overflow_8_to_16, uint64_t * overflow_16_to_64, size_t n );

/* Measured integer ALU-pipe ceiling of the current device: the rate of the
 * fused packed 16x2 add-max instruction, in operations per second (an add and
 * a max in each 16-bit half of each thread: 4 per instruction and thread),
 * and the same as warp instructions per clock per SM.  The denominator of the
 * search kernels' integer-pipe roofline.  Returns 0 on success. */
int ssa_b200_int_peak( double * lane_ops_per_second, double * instructions_per_clock_per_sm );

/* Issue rate of one packed-integer intrinsic on the current device, in warp
 * intrinsics per clock per SM (eight interleaved dependent chains on every SM):
 * op 0 __viaddmax_s16x2, 1 __vmaxs2, 2 __vimax3_s16x2, 3 __vaddss2,
 * 4 __vsubss2, 5 __vaddss4, 6 __vmaxs4, 7 __vsubus4, 8 __vaddus4, 9 __vmaxu4,
 * 10 __vadd4, 11 __vsub4, 12 max.f16x2, 13 32-bit integer add.  The
 * measurement behind the choice of 16x2 lanes
 * over 8x4 ones.  Returns 0, or -1 for an unknown op or a CUDA error. */
int ssa_b200_simd_rate( int op, double * per_clock_per_sm );

/*
 * Database-sharded search, for one process per GPU.  No counterpart in the
 * reference, whose threads split a search by database chunk
 * (src/algo/manager.c:83-185, chunks from src/db_adapter.c:212-239) inside one
 * process.  Every process loads the same database through the plugin; each
 * scores its own contiguous range of records, and one process gathers the
 * per-record results and replays them.
 *
 * ssa_b200_shard_scores: the entry pass and overflow cascade of every query
 * against records [id_lo, id_hi) only.  For query q and record id the arrays
 * (n_queries x (id_hi - id_lo), row-major, index q * (id_hi - id_lo) + id -
 * id_lo) receive the pair's final score, and the number of 4-column blocks the
 * entry-width lane and the 16-bit lane spent on it where they overflowed
 * (-1 where the lane reported; empty records: 0, -1, -1).
 *
 * ssa_b200_replay_gathered: given those arrays for ALL records (n_queries x
 * database size, gathered from every range in record order), replays the
 * reference's lane schedule and top-hit heap per query and, for
 * COMPUTE_ALIGNMENT, traces the hits back on this process's device.
 * results[i] is exactly the list sw_align/nw_align returns for queries[i];
 * with COMPUTE_SCORE it needs no device.
 *
 * Both take amino-acid queries, or nucleotide queries on the forward strand,
 * with the current global settings, and return 0, or -1 (message on stderr)
 * for other setups or bad arguments.
 */
int ssa_b200_shard_scores( int algorithm, p_query * queries, size_t n_queries, int bit_width, size_t id_lo,
        size_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16 );
int ssa_b200_replay_gathered( int algorithm, p_query * queries, size_t n_queries, size_t hitcount, int bit_width,
        int align_type, const int64_t * scores, const int32_t * blocks_entry, const int32_t * blocks_16,
        p_alignment_list * results );

/*
 * Entry-pass shape table.  The entry kernels pick their tile shape (rows per
 * thread and resident CTAs per SM of the query-pair kernel; threads per
 * sequence and rows per thread of the single-query kernel) per query from
 * measured costs per shape and database bucket, written by libssa_b200/tune.py
 * into libssa_b200/tuning/b200.tune (SSA_B200_TUNING=<path> reads another
 * file, SSA_B200_TUNING=builtin the built-in costs).  This writes, as
 * NUL-terminated JSON, where the table came from (file, version, device) and
 * the shapes the last search call ran with; returns the length needed
 * including the NUL.  The reference has a fixed tile instead
 * (src/algo/8/search_8_util.h:25-27). */
size_t ssa_b200_tuning_report( char * buf, size_t n );

/* Marks the packed copy of the database stale, so the next search reads it
 * again through the plugin.  init_db() does this itself; call it after
 * loading a database into the plugin by other means. */
void ssa_db_refresh( void );

/* Number of residue codes of a query after mapping. */
size_t ssa_query_length( p_query p );

/* Translation table of NCBI genetic code `code` (1-6, 9-16, 21-25) as
 * translated searches use it: out[a*256 + b*16 + c] is the amino-acid code of
 * the nucleotide triple (a, b, c), nucleotide codes 0-15 (IUPAC bit masks).
 * Returns 0, or -1 for a code that does not exist. */
int ssa_b200_translation_table( int code, uint8_t * out );

/*
 * Database plugin extension implemented by libsdb_b200 (the plugin that ships
 * with this library): installs count records from memory, record i being
 * residues[offsets[i] .. offsets[i+1]).  The data is copied.  Returns 0.
 */
int ssa_db_b200_load_memory( size_t count, const char * residues, const uint64_t * offsets );

/*
 * Serving.  No counterpart in the reference, which searches one query per call.
 *
 * A server keeps the database and `slots` query slots resident on the device
 * and runs a request loop on its own thread: arriving queries are admitted into
 * free slots (first come, first served, while the traceback memory of the
 * admitted requests stays within `memory_budget` bytes; 0 = no limit) and
 * folded into the running scan of the database, which proceeds in `segments`
 * waves, each covering one segment for every occupied slot; a request is done
 * after one full turn of the segments.  Each result equals what sw_align (or
 * nw_align) returns for the query alone with the settings current at
 * ssa_server_start (matrix, gaps, symbol type, chunk size, SIMD schedule),
 * whatever else is in flight.  submit/wait may be called from any thread;
 * other searches may run meanwhile (they take turns with the server's waves).
 * The database must not change while a server runs.  A query must stay valid
 * until its result list is freed with free_alignment (the list borrows the
 * query's residues, as in sw_align).  Queries are limited to
 * SSA_B200_SERVE_MAX_QUERY residues; submit returns -1 for longer ones.
 */
#define SSA_B200_SERVE_MAX_QUERY 8192u

typedef struct ssa_server ssa_server;

typedef struct {
    uint64_t submitted, completed;
    uint64_t waves;              /* segment waves run so far */
    uint64_t cells;              /* query length x database residues of completed requests */
    double busy_seconds;         /* wall time of the loop's waves and completions */
    double device_seconds;       /* device time of the waves' entry passes and cascades */
    uint32_t slots, segments;
    uint64_t queued;             /* requests not admitted at the first wave after their submit */
    uint64_t slot_waves;         /* occupied slots summed over waves (mean occupancy = slot_waves / waves) */
    uint32_t max_pending;        /* most requests waiting for admission after an admission point */
    uint32_t max_occupied;       /* most slots occupied in one wave */
} ssa_server_stats_t;

ssa_server * ssa_server_start( int algorithm, size_t hitcount, int bit_width, int align_type, size_t slots,
        size_t segments, size_t memory_budget );
/* Returns the request's ticket (>= 0), or -1. */
long long ssa_server_submit( ssa_server * server, p_query query );
/* Blocks until the request is done; returns its list (free with free_alignment)
 * and, if latency_seconds is not NULL, the time from submit to completion. */
p_alignment_list ssa_server_wait( ssa_server * server, long long ticket, double * latency_seconds );
void ssa_server_get_stats( ssa_server * server, ssa_server_stats_t * out );
/* Finishes every submitted request, frees the results nobody waited for, and
 * releases the server. */
void ssa_server_stop( ssa_server * server );

/*
 * Allocation-free scoring.  No counterpart in the reference, whose searches
 * allocate their buffers per call (src/algo/searcher.c:43,160).
 *
 * Scores one query against count database sequences that the caller already
 * holds in device memory, as a BIT_WIDTH_64 search scores them (same scores as
 * sw_align/nw_align at BIT_WIDTH_64), writing d_scores[i] for sequence i.
 * Uses the global matrix and gap penalties.  Within the limits below (and
 * score-table entries within int16, else SSA_B200_NOALLOC_EINVAL) every value
 * of the recurrence stays below 2^29 in magnitude, so the int32 arithmetic
 * and int32 scores are exact.
 * Residues are the library's codes: index into "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"
 * for amino acids, into "-ACMGRSVTWYHKDBN" for nucleotides; sequence i is
 * d_db_codes[d_db_offsets[i] .. + d_db_lengths[i]).  A sequence of length 0
 * scores 0.
 *
 * It allocates no memory: for callers whose device memory is reserved by
 * their own pool, or that cannot take cudaFree's device-wide synchronisation
 * on a latency-bound path.  Its working buffers are fixed-size device arrays
 * of the library (about 9.6 MiB per device), set up by the first call on each
 * device, which also loads every kernel the call uses -- make that first call,
 * with the device current, before the phase that must not allocate and before
 * any stream capture.  Calls must be made in the device's primary context
 * (the one the CUDA runtime API uses).  Sizes beyond the
 * limits below are rejected with SSA_B200_NOALLOC_ETOOBIG; max_seq_len is the
 * caller's bound on the database lengths.  The call runs on `stream` (a
 * cudaStream_t; NULL = default stream) and returns when the scores are
 * written.  Calls overlapping in time on one device (two host threads, or two
 * streams) share the buffers and race.
 */
#define SSA_B200_NOALLOC_MAX_QUERY 4096u
#define SSA_B200_NOALLOC_MAX_SEQ_LEN 4096u
#define SSA_B200_NOALLOC_MAX_SEQS 262144u

#define SSA_B200_NOALLOC_OK 0
#define SSA_B200_NOALLOC_EINVAL 1      /* bad argument or no score matrix */
#define SSA_B200_NOALLOC_ETOOBIG 2     /* a size above the limits above */
#define SSA_B200_NOALLOC_ECUDA 3       /* CUDA error */
#define SSA_B200_NOALLOC_ESEQLEN 4     /* a sequence exceeded SSA_B200_NOALLOC_MAX_SEQ_LEN */

int ssa_b200_score64_noalloc( int algorithm, const uint8_t * d_query, uint32_t query_len,
        const uint8_t * d_db_codes, const uint64_t * d_db_offsets, const uint32_t * d_db_lengths, uint32_t count,
        uint32_t max_seq_len, int32_t * d_scores, void * stream );

#ifdef __cplusplus
}
#endif

#endif /* LIBSSA_B200_H_ */
