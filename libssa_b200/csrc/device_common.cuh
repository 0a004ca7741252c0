// device_common.cuh -- data structures shared by the host engine and the
// sm_100a kernels of the libssa B200 build.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

namespace ssa {

// One (query, database sequence) unit of work of a saturating pass.  nb is
// the number of 4-column blocks the sequence occupied in the previous pass
// (its lane-schedule length there); 0 for the entry pass.
struct PairTask {
    uint32_t qslot;
    uint32_t id;
    int32_t nb_prev;
    int32_t pad_;
};

// Device view of the packed database.  Codes are stored per sequence in ID
// order; each sequence is followed by zero codes up to a multiple of 16 bytes.
struct DbView {
    const uint8_t * codes;
    const uint64_t * offsets;     // per ID
    const uint32_t * lens;        // per ID (0 = empty record, never searched)
    uint32_t n_ids;
};

// Per-query data of a batch.  prof32 holds, for every query slot, the
// 32 x qpad table prof[code][row] of substitution scores at the pass width
// (matrix[(code << 5) + query[row]] truncated to 8 or 16 bits, or exact).
struct QueryView {
    const int32_t * prof32;
    const uint64_t * prof32_off;  // per slot, in elements
    const uint32_t * qlen;        // per slot
    const uint32_t * qpad;        // per slot, rows of the profile
    uint32_t n_slots;
    // the same table with exact int64 entries (same offsets), for the 64-bit
    // pass in int64 arithmetic; nullptr otherwise
    const int64_t * prof64 = nullptr;
};

// Result sink of a pass.  score[slot * n_ids + id] receives the pass's score.
// Sequences the pass does not report (overflow, or a score outside the
// reportable range) are appended to next[] with the block count they used.
struct PassSink {
    int32_t * score;
    uint64_t score_stride;        // = n_ids
    PairTask * next;
    unsigned int * next_count;
    uint32_t next_cap;
    unsigned int * error_flags;   // bit 0: next[] overflow
    // the 64-bit pass in int64 arithmetic writes its scores here (same index)
    // and SCORE_IN_WIDE into score[]
    int64_t * score64 = nullptr;
};

// score[] marker of a pair whose exact score is in PassSink::score64
constexpr int32_t SCORE_IN_WIDE = INT32_MIN;

enum ErrorBits : unsigned int {
    ERR_REQUEUE_OVERFLOW = 1u,
    ERR_SCRATCH_OVERFLOW = 2u,
    ERR_PIPELINE = 4u,            // a stripe pipeline ran past its step bound
};


// Parameters of the saturating-lane emulation kernel (emul_kernel.cu).
struct EmulParams {
    DbView db;
    QueryView qv;
    const PairTask * tasks;     // explicit task list, or nullptr
    const uint32_t * order;     // implicit tasks: non-empty IDs, longest first
    const uint32_t * slot_list; // implicit tasks over these slots (nullptr: all slots)
    uint32_t n_sub;             // entries of slot_list
    uint64_t n_tasks;
    unsigned long long * counter;
    int gap_open, gap_extend;
    PassSink sink;
    int4 * scratch;             // per warp: scratch_cols entries
    uint32_t scratch_cols;
};

// Traceback work item and result (traceback_kernels.cu).
struct TbHit {
    uint32_t qslot;
    uint32_t id;
    int32_t score;      // search score
    int32_t algo;       // 0 SW, 1 NW
};

struct TbRegion {
    int32_t a_begin, a_end;   // query rows
    int32_t b_begin, b_end;   // database columns
    int32_t fwd_score;        // SW: forward-pass maximum; NW: H(a_end, b_end) from the direction pass
    // layout of the hit's direction words: words per column (query rows / 8,
    // rounded up) and the first database column stored
    int32_t dir_words, dir_col0;
    int32_t status;           // 0 ok, 1 no positive cell, 2 reverse pass found nothing
};

// Query rows per 16-bit direction word (2 bits per cell).
constexpr int TB_WORD_ROWS = 8;

struct TbParams {
    DbView db;
    const uint8_t * qcodes;     // per slot
    const uint64_t * qoff;
    const uint32_t * qlen;
    const int64_t * matrix;     // 32x32 [(row << 5) + col]
    int gap_open, gap_extend;
    const TbHit * hits;
    uint32_t n_hits;
    TbRegion * regions;
    int4 * scratch;             // per group of warps on one hit
    uint32_t scratch_cols;
    int32_t * last_h;           // per hit: forward pass last-row H (query-indexed)
    int32_t * last_e;           // per hit: forward pass last-row vertical gap
    const uint64_t * last_off;  // per hit offset into last_h / last_e
    uint16_t * dirs;            // per hit direction words
    const uint64_t * dir_off;   // per hit offset into dirs
    char * ops;                 // per hit reversed op string
    const uint64_t * ops_off;
    uint32_t * ops_len;
    unsigned int * error_flags;
    unsigned long long * hit_counters;   // forward, reverse, directions: next hit to take (start at 0)
};

// Kernel launchers.
// wide: the 64-bit pass in int64 arithmetic (p.qv.prof64, p.sink.score64,
// scratch of 32 bytes per column); otherwise int32
cudaError_t launch_emul( int algo, int width, const EmulParams & p, int grid, cudaStream_t st, bool wide = false );
cudaError_t launch_build_profile32( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int width, int32_t * prof,
        uint32_t n_slots, cudaStream_t st );
// loads the int32 64-bit lane kernels and the int32 profile builder onto the
// current device (no launch)
cudaError_t preload_emul64();
// exact int64 entries, layout of launch_build_profile32
cudaError_t launch_build_profile64( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int64_t * prof, uint32_t n_slots,
        cudaStream_t st );
// group: warps per hit, 1, 2 or 4 (scratch: one boundary row per group)
cudaError_t launch_tb_regions( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev );
cudaError_t launch_tb_paths( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev );
cudaError_t launch_tb_fused( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev );


// ---- fast Smith-Waterman entry pass (sw_fast_kernel.cu) --------------------
// Residue code used after a sequence's last 4-column block in the pair layout;
// its profile row is -128, so it never changes a Smith-Waterman maximum.
constexpr uint32_t FAST_PAD_CODE = 31;

struct FastParams {
    const uint8_t * pair_res;     // per pair: cols x (residue A, residue B)
    const uint64_t * pair_off;    // byte offset of each pair (16-aligned)
    const uint32_t * pair_cols;   // columns of each pair, a multiple of 8
    const uint2 * pair_ids;       // database IDs (B = 0xffffffff when absent)
    const int8_t * prof8;         // per slot: 32 x rows int8 scores
    const uint64_t * prof8_off;   // per slot, bytes
    const uint16_t * slot_group;  // per slot: threads per pair G
    const uint32_t * slot_rows;   // per slot: profile rows (passes x G x R)
    // work units u = chunk * n_class + i: slot unit_slots[i] against pairs
    // [chunk_bounds[chunk], chunk_bounds[chunk + 1])
    const uint32_t * unit_slots;
    uint32_t n_class;
    const uint32_t * chunk_bounds;
    uint64_t n_units;
    unsigned long long * unit_counter;
    int gap_oe;                   // (int8) (gapO + gapE)
    int gap_e;
    PassSink sink;
    int4 * scratch;               // per warp and group slot (4 per warp, 8 for the 4-column kernel): scratch_cols entries
    uint32_t scratch_cols;
    uint32_t slice_rows;          // largest G x R of the launch: rows of a warp's profile slice
};

constexpr int FAST_THREADS = 128;   // threads per CTA of the fast pass

cudaError_t launch_sw_fast( int R, const FastParams & p, int grid, cudaStream_t st, int * blocks_per_sm );
// the same pass with one 4-column block per step (G = 4, 8, 16 or 32; scratch
// rows for 8 groups per warp)
cudaError_t launch_sw_fast4( int R, const FastParams & p, int grid, cudaStream_t st, int * blocks_per_sm );
cudaError_t launch_build_profile8( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * slots, uint32_t n, const uint32_t * rows_of, const int64_t * matrix, int8_t * prof,
        const uint64_t * prof_off, cudaStream_t st );

// ---- query-pair Smith-Waterman entry pass (sw_qpair_kernel.cu) -------------
// Two queries of similar length share each 32-bit register (low half query A,
// high half query B) against one database sequence per group of QP_G threads.
constexpr int QP_G = 4;               // threads per sequence
constexpr int QP_GPW = 32 / QP_G;     // sequences per warp
constexpr int QP_CODES = 28;          // residue codes with a profile row (AA 0..27, NT 0..15)
constexpr int QP_THREADS_PER_CTA = 128;

struct QPairParams {
    DbView db;
    const uint32_t * order;       // non-empty IDs, longest first
    const uint32_t * prof;        // per query pair: QP_CODES x rows words (16x2: A low, B high)
    const uint64_t * prof_off;    // per query pair, in words
    const uint32_t * qp_slots;    // per query pair: slot A, slot B (0xffffffff when absent)
    const uint32_t * qp_rows;     // per query pair: profile rows (passes x QP_G x R)
    // work units u = i * n_chunks + chunk: query pair unit_pairs[i] against the
    // sequences order[chunk_bounds[chunk] .. chunk_bounds[chunk + 1]); the
    // pairs come longest first, so the longest units start first
    const uint32_t * unit_pairs;
    uint32_t n_class;
    uint32_t n_chunks;
    const uint32_t * chunk_bounds;
    uint64_t n_units;
    unsigned long long * unit_counter;
    int gap_oe;                   // (int8) (gapO + gapE)
    int gap_e;
    PassSink sink;
    int4 * scratch;               // per warp and group: scratch_cols column pairs (H, F of two columns)
    uint32_t scratch_cols;
    // Needleman-Wunsch only (nw_qpair_kernel)
    int gap_open;
    const uint32_t * qlen;        // per slot
    const uint32_t * qp_lmax;     // per query pair: longest sequence the kernel scores exactly
    PairTask * redo;              // longer sequences: (slot, id) for the lane emulation
    unsigned int * redo_count;
    uint32_t redo_cap;
};

// mb: 4 or 5 resident CTAs per SM (register bound of the instantiation)
cudaError_t launch_sw_qpair( int R, int mb, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm );
// the same pass with one 4-column block per step (four dependency chains per
// thread); hmax: the running maximum in fp16x2 off the ALU pipe (mb 4 only);
// g8: R = 24 rows per pass of 4 threads run as 8 threads of 12 rows
cudaError_t launch_sw_qpair4( int R, int mb, bool hmax, bool g8, const QPairParams & p, int grid, cudaStream_t st,
        int * blocks_per_sm );
cudaError_t launch_nw_qpair( int R, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm );
// the same pass with one 4-column block per step (four dependency chains per thread)
cudaError_t launch_nw_qpair4( int R, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm );
// width 8: (int8) scores, -128 past a query (Smith-Waterman 8-bit entry);
// width 16: (int16) scores, 0 past a query (Needleman-Wunsch 16-bit entry)
cudaError_t launch_build_profile_qp( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qp_slots, uint32_t n_qp, const uint32_t * qp_rows, const int64_t * matrix, uint32_t * prof,
        const uint64_t * prof_off, int width, cudaStream_t st );

// ---- long pairs (pair_kernel.cu) ---------------------------------------------
// A group of PAIR_W warps scores one (query, database sequence) pair exactly in
// int32: lane k of a warp owns PAIR_R query rows of a stripe of 32 x PAIR_R rows.
constexpr int PAIR_R = 16;
constexpr int PAIR_W = 4;
constexpr int PAIR_THREADS = 256;

struct PairScoreParams {
    DbView db;
    const uint8_t * qcodes;       // per query slot: codes at qoff[slot]
    const uint64_t * qoff;
    const uint32_t * qlen;
    const uint32_t * pair_slot;   // per pair, in work order (largest first): query slot
    const uint32_t * pair_unit;   // per pair: database unit
    uint32_t n_pairs;
    const int64_t * matrix;       // 32 x 32, [database code][query code]
    int gap_open, gap_extend;
    int32_t * score;              // per pair, in work order
    int4 * scratch;               // per group of PAIR_W warps: scratch_cols boundary columns (H, F)
    uint32_t scratch_cols;
    unsigned long long * counter;
    unsigned * error_flags;
};

cudaError_t launch_pair_score( int algo, const PairScoreParams & p, int grid, cudaStream_t st, int * blocks_per_sm );

}  // namespace ssa
