/*
 * ssa_oracle.h -- CPU restatement of the libssa database-search path.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle the CUDA build is compared against.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it.  It is itself pinned against the reference binary built from the
 * reference's sources (oracle/_ref/ref_run) and the reference's known-answer
 * tests.  Every function cites the reference lines it restates.
 *
 * Sequences are passed as mapped residue codes (0..31); the score matrix is
 * the reference's 32x32 int64 table indexed [(row << 5) + col].
 */
#ifndef SSA_ORACLE_H_
#define SSA_ORACLE_H_

#include <stdint.h>
#include <stddef.h>

typedef struct {
    int algo;               /* 0 = Smith-Waterman, 1 = Needleman-Wunsch */
    int bit_width;          /* entry width of the cascade: 8, 16 or 64 */
    int align_type;         /* 0 = COMPUTE_SCORE, 1 = COMPUTE_ALIGNMENT */
    int lanes8;             /* channels of the 8-bit pass (32 AVX2, 16 SSE4.1) */
    int lanes16;            /* channels of the 16-bit pass (16 AVX2, 8 SSE2) */
    int gap_open;           /* negative, int8 range */
    int gap_extend;         /* negative, int8 range */
    uint64_t hitcount;
    uint64_t chunk_size;
    int64_t matrix[1024];
} oracle_config;

typedef struct {
    int64_t score;
    uint64_t id;
    uint64_t q_start, q_end, d_start, d_end;
    char * cigar;           /* malloc'd; NULL for COMPUTE_SCORE */
} oracle_hit;

typedef struct {
    uint64_t overflow8;     /* sequences re-aligned at 16 bit */
    uint64_t overflow16;    /* sequences re-aligned at 64 bit */
} oracle_stats;

/* Result of one database sequence in one lane of a saturating pass. */
typedef struct {
    int64_t score;          /* reported score (valid when !overflow) */
    int overflow;           /* 1 if the lane overflowed */
    int64_t blocks;         /* 4-column blocks the lane spent on the sequence */
} oracle_lane;

#ifdef __cplusplus
extern "C" {
#endif

/* Full search: chunking, cascade, lane schedules, heap, sort, traceback. */
int oracle_search( const oracle_config * cfg, const uint8_t * query, uint64_t qlen, uint64_t n_db,
        const uint8_t * db, const uint64_t * offsets, oracle_hit * out, uint64_t * out_len, oracle_stats * stats );

void oracle_free_hits( oracle_hit * hits, uint64_t n );

/* One sequence through one saturating pass, as if alone in its lane. */
oracle_lane oracle_lane_result( const oracle_config * cfg, int width, const uint8_t * query, uint64_t qlen,
        const uint8_t * dseq, uint64_t dlen );

/* Exact scalar scores (reference: src/algo/64/smith_waterman_63.c:32-98,
 * src/algo/64/needleman_wunsch_64.c:32-98). */
int64_t oracle_full_sw( const oracle_config * cfg, const uint8_t * dseq, uint64_t dlen, const uint8_t * q,
        uint64_t qlen );
int64_t oracle_full_nw( const oracle_config * cfg, const uint8_t * dseq, uint64_t dlen, const uint8_t * q,
        uint64_t qlen );

/* Traceback of one pair: region, CIGAR (malloc'd) and coordinates. */
int oracle_align_pair( const oracle_config * cfg, const uint8_t * q, uint64_t qlen, const uint8_t * d, uint64_t dlen,
        uint64_t * q_start, uint64_t * q_end, uint64_t * d_start, uint64_t * d_end, char ** cigar );

/* Residue mapping.  nucleotide selects the NCBI nt16 alphabet, otherwise the
 * NCBI amino-acid alphabet.  drop_unknown=1 removes unmapped symbols (query
 * rule), 0 maps them to code 0 (database rule).  Returns the output length. */
uint64_t oracle_map( const char * ascii, uint64_t n, int nucleotide, int drop_unknown, uint8_t * out );

/* Parses score-matrix text into the 32x32 table (-1 where unset). */
int oracle_parse_matrix( const char * text, int64_t * out );

/* Constant match/mismatch table. */
void oracle_constant_matrix( int match, int mismatch, int64_t * out );

#ifdef __cplusplus
}
#endif

#endif /* SSA_ORACLE_H_ */
