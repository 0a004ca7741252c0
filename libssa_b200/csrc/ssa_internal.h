// ssa_internal.h -- internal interfaces of the libssa B200 library.
#pragma once

#include <climits>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "libssa.h"

namespace ssa {

// ---- process-global settings (reference: src/libssa.c:35-36,
//      src/util/util.c:34, src/algo/manager.c:38, src/util/util_sequence.c) ----
struct Config {
    int output_mode = OUTPUT_WARNING;
    int simd_mode = COMPUTE_ON_AVX2;
    size_t chunk_size = 1000;
    size_t thread_count = (size_t) -1;
    int8_t gap_open = 0;
    int8_t gap_extend = 0;
    int symtype = AMINOACID;
    int strands = FORWARD_STRAND;
    int db_gencode = 1;
    int q_gencode = 1;
    bool matrix_set = false;
    bool constant_scoring = false;
    int64_t matrix[1024];
};

Config & config();

[[noreturn]] void fatal( const char * fmt, ... );
void print_info( const char * fmt, ... );
void print_warning( const char * fmt, ... );
void print_error( const char * fmt, ... );

// ---- residue maps (reference: src/util/util_sequence.c:38-88) ----------------
int map_aa( unsigned char c );     // -1 if not an amino-acid symbol
int map_nt16( unsigned char c );   // -1 if not a nucleotide symbol

// ---- matrices (reference: src/matrices.c:335-568) ----------------------------
void matrix_from_string( const char * text, int64_t * out );
bool matrix_builtin( const char * name, int64_t * out );
void matrix_constant( int match, int mismatch, int64_t * out );

// ---- database packed on the host, mirrored into HBM --------------------------
// The database as the searches see it: units.  A record (database ID) gives
// `upi` consecutive units, unit id * upi + k: its mapped residues (k = 0) and,
// for nucleotide searches of the complementary strand, their reverse
// complement (k = 1), as the reference's chunks hold them
// (src/db_adapter.c:47-70, 118-135, 212-239).  The per-unit arrays below say
// "ID" for the unit index; with upi = 1 units are records.
struct HostDb {
    uint32_t n_ids = 0;                 // units
    uint32_t n_records = 0;             // database IDs
    uint32_t upi = 1;                   // units per record
    std::vector<uint32_t> len;          // per ID
    std::vector<uint64_t> off;          // per ID into codes
    std::vector<uint8_t> codes;         // mapped residues, each record padded to 16 B
    std::vector<uint32_t> order_desc;   // non-empty IDs, longest first (stable)
    std::vector<uint32_t> nonempty_before;   // per ID + 1: non-empty records with a smaller ID
    // length-sorted pairs for the 16x2 Smith-Waterman pass: IDs and padded
    // column counts (the interleaved residues live only in HBM)
    std::vector<uint32_t> pair_cols;
    std::vector<uint32_t> pair_a, pair_b;   // pair_b = 0xffffffff when absent
    double mean_len = 0;
    uint64_t residues = 0;
    uint32_t max_len = 0;
    int symtype = -1;
    int strands = -1;
    uint64_t generation = 0;
};

// units per record for the current settings
uint32_t units_per_record( int symtype, int strands );
uint8_t nt_complement( uint8_t x );

// ---- hits and search requests -------------------------------------------------
struct Hit {
    int64_t score = 0;
    uint32_t id = 0;            // database record (ID)
    uint32_t unit = 0;          // database unit (record x units per record + strand)
    uint32_t q_index = 0;       // strand or frame of the query (its search order)
    uint8_t db_strand = 0, db_frame = 0;
    uint32_t q_start = 0, q_end = 0, d_start = 0, d_end = 0;
    std::string cigar;
    bool has_cigar = false;
};

struct SearchStats {
    uint64_t overflow8 = 0;     // sequences re-aligned at 16 bit
    uint64_t overflow16 = 0;    // sequences re-aligned at 64 bit
    // the same per query (per entry of the call's query list)
    std::vector<std::pair<uint64_t, uint64_t>> query_overflow;
    uint64_t cells = 0;         // query length x database residues, summed
    uint64_t kernel_launches = 0;
    double seconds_gpu = 0;
    double entry_seconds = 0;
    double kernel_seconds = 0;
    uint64_t h2d_bytes = 0;
    uint64_t d2h_bytes = 0;
};

struct SearchRequest {
    int algo = 0;               // 0 SW, 1 NW
    int bit_width = 8;
    int align_type = COMPUTE_SCORE;
    size_t hitcount = 10;
    size_t chunk_size = 1000;
    int lanes8 = 32, lanes16 = 16;
    int gap_open = 0, gap_extend = 0;
    const int64_t * matrix = nullptr;
};

struct QueryCodes {
    const uint8_t * codes;
    uint32_t len;
};

// Runs the search of each query against the current database on the GPU and
// returns the sorted hit list per query.  groups[g] consecutive entries of
// `queries` are the strands or frames of query g, merged into one hit list
// (empty groups: one entry per query).
void engine_search( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & groups, std::vector<std::vector<Hit>> & out, SearchStats & stats );

// The packed database (re-read through the plugin when stale).
// Query i against database unit units[i] alone (one hit per pair, none for an
// empty sequence); the hits carry alignments when req.align_type asks for them.
void engine_align_pairs( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & units, std::vector<std::vector<Hit>> & out, SearchStats & stats );
// Device memory for the direction words of one traceback wave (0 = automatic).
void engine_set_traceback_memory( uint64_t bytes );
// Device memory for the database (0 = automatic); a database that does not fit
// is streamed through the device in segments.
void engine_set_db_memory( uint64_t bytes );
// Whether the current database is streamed (packs it first if needed).
bool engine_streaming();
const HostDb & engine_database();
void engine_invalidate_database();
void engine_shutdown();
uint64_t engine_kernel_launches();

// ---- database-sharded searches ------------------------------------------------
// Entry pass and cascade of every query against database records [id_lo,
// id_hi) only: scores[q * (id_hi - id_lo) + id - id_lo] = the pair's final
// score, blocks_entry / blocks_16 = the blocks the entry-width / 16-bit lane
// spent where it overflowed, else -1 (empty records: 0, -1, -1).
void engine_shard_scores( const SearchRequest & req, const std::vector<QueryCodes> & queries, uint32_t id_lo,
        uint32_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16, SearchStats & stats );
// Traceback of replayed hit lists (out[q] belongs to queries[q]).
void engine_align_hits( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        std::vector<std::vector<Hit>> & out, SearchStats & stats );
// The record lengths of the plugin's database (host only, no device).
void lengths_db( HostDb & db );

// ---- measured entry-pass shape costs (tuning.cpp, libssa_b200/tune.py) ---------
constexpr int TUNE_BUCKETS = 6;   // database mean length <250 / <1000 / longer, x fewer / more than 50,000 sequences

struct TuningTable {
    int version = 0;
    std::string device;
    std::string source = "built-in";
    // query-pair kernel: cost per (query pair, pass, database column) by
    // [bucket][R / 4 - 4][resident CTAs per SM - 4][variant: 2 columns per
    // step, 4 columns, 4 columns with the running maximum in fp16x2, 4 columns
    // with 8 threads per sequence (R = 24 only)]; 0 = not measured
    double qpair[TUNE_BUCKETS][4][2][4] = {};
    // single-query kernel: cost per (pass, database column) by
    // [bucket][G = 8, 16, 32][R / 8 - 1]; 0 = not measured
    double fast[TUNE_BUCKETS][3][4] = {};
    bool has_fast = false;
    // the same for its 4-column variant: [bucket][G = 4, 8, 16, 32][R / 8 - 1]
    double fast4[TUNE_BUCKETS][4][4] = {};
    bool has_fast4 = false;
};

const TuningTable & tuning();
int db_bucket( double mean_len, uint64_t n_seqs );
// JSON of the table's origin and the shapes the last search call used
std::string tuning_report();

// ---- host replay of the CPU lane schedule and min-heap (replay.cpp) ----------
// score[] marker of a pair whose exact score is in ReplayQuery::score64 (the
// 64-bit pass ran in int64 arithmetic)
constexpr int32_t REPLAY_SCORE_IN_WIDE = INT32_MIN;

struct ReplayQuery {
    const int32_t * score = nullptr;                // per ID, final score
    const int64_t * score64 = nullptr;              // per ID, where score[] holds the marker
    std::vector<std::pair<uint32_t, int32_t>> ovf_entry;   // (id, blocks) not reported by the entry pass
    std::vector<std::pair<uint32_t, int32_t>> ovf16;       // (id, blocks) not reported by the 16-bit pass

    int64_t score_of( uint32_t id ) const {
        const int32_t s = score[id];
        return (s == REPLAY_SCORE_IN_WIDE && score64) ? score64[id] : (int64_t) s;
    }
};

// ---- serving (engine.cu): resident query slots, waves over database segments --
constexpr uint32_t SERVE_MAX_QUERY = 8192;   // residues of a served query

struct ServeOverflow {
    uint32_t slot, id;
    int32_t nb;      // blocks the lane spent on the sequence in that pass
};

// Sets up `slots` resident query slots for requests of `req`'s kind; returns the
// bounds of `segments` ranges of the length-sorted non-empty sequences.
std::vector<uint32_t> engine_serve_open( const SearchRequest & req, uint32_t slots, uint32_t segments );
void engine_serve_load( uint32_t slot, const uint8_t * codes, uint32_t len );
// Entry pass and cascade of the `active` slots over sequences [seq_lo, seq_hi).
void engine_serve_wave( const SearchRequest & req, const std::vector<uint32_t> & active, uint32_t seq_lo,
        uint32_t seq_hi, std::vector<ServeOverflow> & ovf_entry, std::vector<ServeOverflow> & ovf16,
        SearchStats & stats );
// Replay, heap and traceback of finished slots; out is indexed by slot.
void engine_serve_finish( const SearchRequest & req, const std::vector<uint32_t> & done,
        std::vector<ReplayQuery> & rq, std::vector<std::vector<Hit>> & out, SearchStats & stats );

// Chunk schedule ranks that do not depend on the query (entry pass without
// overflow): rank[id] = report position of id inside its chunk.
struct ScheduleCache {
    size_t chunk_size = 0;
    int lanes = 0;
    uint64_t generation = 0;
    std::vector<uint32_t> rank;
};

void schedule_ranks( const HostDb & db, size_t chunk_size, int lanes, std::vector<uint32_t> & rank );

struct ReplayCounts {
    uint64_t overflow8 = 0;     // searched sequences the 8-bit pass re-queued
    uint64_t overflow16 = 0;    // searched sequences re-queued to 64 bit
};

void replay_frames( const HostDb & db, const SearchRequest & req, const ReplayQuery * rq, uint32_t F,
        std::vector<Hit> & hits, ReplayCounts & counts );
void replay_query( const HostDb & db, const SearchRequest & req, const ReplayQuery & rq, const uint32_t * rank_entry,
        std::vector<Hit> & hits, ReplayCounts & counts );

}  // namespace ssa
