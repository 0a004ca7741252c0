/*
 * libssa.h -- public C API of the B200 libssa build.
 *
 * This header is a drop-in for the CPU libssa API (reference: src/libssa.h).
 * Every constant, struct layout and function signature below is the same as
 * the reference's, so a program compiled against the CPU library links
 * against this one unchanged.  Behind the boundary the database is packed into
 * HBM once per init_db() and the search, overflow cascade and traceback run as
 * sm_100a CUDA kernels; there is no CPU fallback.
 *
 * Each declaration cites the reference declaration it replaces.
 */
#ifndef LIBSSA_H_
#define LIBSSA_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants (reference: src/libssa.h:29-72) -------------------------- */
#define VERBOSE_ON 1
#define VERBOSE_OFF 0

#define SIMD_ON 1
#define SIMD_OFF 0

#define BLOSUM45 "blosum45"
#define BLOSUM50 "blosum50"
#define BLOSUM62 "blosum62"
#define BLOSUM80 "blosum80"
#define BLOSUM90 "blosum90"
#define PAM30 "pam30"
#define PAM70 "pam70"
#define PAM250 "pam250"

#define NUCLEOTIDE 0
#define AMINOACID 1
#define TRANS_QUERY 2
#define TRANS_DB 3
#define TRANS_BOTH 4

#define FORWARD_STRAND 1
#define COMPLEMENTARY_STRAND 2
#define BOTH_STRANDS 3

#define BIT_WIDTH_8 8
#define BIT_WIDTH_16 16
#define BIT_WIDTH_64 64

#define OUTPUT_SILENT 0
#define OUTPUT_ERROR 1
#define OUTPUT_WARNING 2
#define OUTPUT_INFO 3

#define COMPUTE_SCORE 0
#define COMPUTE_ALIGNMENT 1

#define READ_FROM_FILE 0
#define READ_FROM_STRING 1
#define MATRIX_BUILDIN 2

#define COMPUTE_ON_SSE2 0
#define COMPUTE_ON_SSE41 1
#define COMPUTE_ON_AVX2 2

/* ---- data types (reference: src/libssa.h:78-117), layouts unchanged ----- */
struct _query;
typedef struct _query * p_query;

typedef struct {
    char* seq;          /* mapped residue codes, owned by the alignment list */
    size_t len;
    size_t ID;          /* 0-based database ID */
    int strand;
    int frame;
} db_seq_t;

typedef struct {
    char* seq;          /* mapped query codes, borrowed from the p_query */
    size_t len;
    int strand;
    int frame;
} q_seq_t;

typedef struct {
    db_seq_t db_seq;
    q_seq_t query;
    char * alignment;   /* NUL-terminated CIGAR, NULL for COMPUTE_SCORE */
    size_t alignment_len;
    long score;
    size_t align_q_start;   /* 0-based, inclusive */
    size_t align_q_end;
    size_t align_d_start;
    size_t align_d_end;
} alignment_t;
typedef alignment_t * p_alignment;

typedef struct {
    p_alignment* alignments;
    size_t len;
} alignment_list_t;
typedef alignment_list_t * p_alignment_list;

/* ---- technical settings (reference: src/libssa.h:122-128) --------------- */

/* Message verbosity: OUTPUT_SILENT .. OUTPUT_INFO (reference: src/libssa.c:41-43). */
void set_output_mode( int mode );

/* Selects which CPU lane schedule the hit order reproduces: COMPUTE_ON_AVX2
 * (32 lanes at 8 bit, 16 at 16 bit), COMPUTE_ON_SSE41 (16/8) or
 * COMPUTE_ON_SSE2 (8-bit search unavailable there, as in the reference).
 * Reference: src/libssa.c:45-47, src/cpu_config.c:29-33. */
void set_simd_compute_mode( int mode );

/* Number of database sequences per chunk; 0 restores the default of 1000
 * with an error message (reference: src/libssa.c:49-56). */
void set_chunk_size( size_t size );

/* Accepted for compatibility; the GPU build runs single-caller and ignores
 * the host thread count (reference: src/libssa.c:58-60). */
void set_thread_count( size_t count );

/* ---- initialisation (reference: src/libssa.h:152-223) ------------------- */

/* mode: READ_FROM_FILE, READ_FROM_STRING or MATRIX_BUILDIN
 * (reference: src/libssa.c:81-94). */
void init_score_matrix( int mode, const char* matrix );

/* Constant scoring.  As in the reference implementation the FIRST argument is
 * the match score and the second the mismatch score
 * (reference: src/libssa.c:115-117 -> src/matrices.c:447). */
void init_constant_scores( const int8_t p, const int8_t m );

/* Negative gap costs: a gap of length k costs gapO + k*gapE
 * (reference: src/libssa.c:102-105). */
void init_gap_penalties( const int8_t gapO, const int8_t gapE );

/* Symbol type, strands and genetic codes (reference: src/libssa.c:139-157). */
void init_symbol_translation( int type, int strands, int db_gencode, int q_gencode );

/* Re-opens the database through the plugin and packs it into HBM on the next
 * search (reference: src/libssa.c:126-132). */
void init_db( const char* db_file );

/* mode: READ_FROM_FILE (first FASTA record) or READ_FROM_STRING
 * (reference: src/libssa.c:165-180). */
p_query init_sequence_fasta( int mode, const char* fasta_seq_file );

/* Frees a query (reference: src/libssa.c:189-191). */
void free_sequence( p_query p );

/* ---- alignment (reference: src/libssa.h:240-262) ------------------------ */

/* Smith-Waterman search of the whole database; returns the top hitcount hits
 * sorted by score then ID, both descending (reference: src/libssa.c:229-235). */
p_alignment_list sw_align( p_query p, size_t hitcount, int bit_width, int align_type );

/* Needleman-Wunsch search (reference: src/libssa.c:245-251). */
p_alignment_list nw_align( p_query p, size_t hitcount, int bit_width, int align_type );

/* Frees a list returned by sw_align/nw_align (reference: src/libssa.c:262-264). */
void free_alignment( p_alignment_list alist );

/* Frees the matrices, closes the database and releases all device memory
 * (reference: src/libssa.c:266-271). */
void ssa_exit( void );

#ifdef __cplusplus
}
#endif

#endif /* LIBSSA_H_ */
