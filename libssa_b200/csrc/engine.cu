// engine.cu -- host orchestration of the GPU search.
//
// One search call (one query through sw_align/nw_align, or a batch through
// the batched extension) runs as:
//
//   1. the database, read once through the libssa_extern_db.h plugin and
//      mapped to residue codes, is resident in HBM (re-packed only after
//      init_db or a change of symbol type);
//   2. the queries of the batch are uploaded and their substitution profiles
//      built on the device, one 32 x rows table per query and pass width;
//   3. the entry pass scores every (query, non-empty sequence) pair; pairs the
//      entry width cannot report go to a device-side re-queue list with the
//      block count they used, and the next width runs on that list
//      (8 -> 16 -> 64, reference: src/algo/8/search_8.c:94-124,
//      src/algo/16/search_16.c:92-114);
//   4. the final score of every pair and the re-queue lists come back to the
//      host, which replays the CPU channel schedule and min-heap per query
//      (replay.cpp) to get the exact CPU hit list;
//   5. for COMPUTE_ALIGNMENT the hits go through the traceback kernels.
#include "device_common.cuh"
#include "ssa_internal.h"
#include "libssa_extern_db.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <thread>
#include <tuple>

namespace ssa {

static_assert( REPLAY_SCORE_IN_WIDE == SCORE_IN_WIDE, "one marker for scores held in int64" );

#define CUDA_CHECK( expr ) \
    do { \
        cudaError_t e_ = (expr); \
        if( e_ != cudaSuccess ) \
            fatal( "CUDA error %s at %s:%d: %s", cudaGetErrorName( e_ ), __FILE__, __LINE__, cudaGetErrorString( e_ ) ); \
    } while( 0 )

// Grow-only device buffer.
struct DevBuf {
    void * p = nullptr;
    size_t bytes = 0;
    void * ensure( size_t n ) {
        if( n > bytes ) {
            if( p )
                CUDA_CHECK( cudaFree( p ) );
            p = nullptr;
            size_t want = std::max( n, (size_t) 256 );
            CUDA_CHECK( cudaMalloc( &p, want ) );
            bytes = want;
        }
        return p;
    }
    void release() {
        if( p )
            cudaFree( p );
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T * as() const {
        return (T *) p;
    }
};

struct PinnedBuf {
    void * p = nullptr;
    size_t bytes = 0;
    void * ensure( size_t n ) {
        if( n > bytes ) {
            if( p )
                CUDA_CHECK( cudaFreeHost( p ) );
            p = nullptr;
            size_t want = std::max( n, (size_t) 256 );
            CUDA_CHECK( cudaMallocHost( &p, want ) );
            bytes = want;
        }
        return p;
    }
    void release() {
        if( p )
            cudaFreeHost( p );
        p = nullptr;
        bytes = 0;
    }
};

class Engine {
public:
    static Engine & get() {
        static Engine e;
        return e;
    }

    void init_device() {
        if( ready_ )
            return;
        int dev = 0;
        if( const char * s = getenv( "SSA_B200_DEVICE" ) )
            dev = atoi( s );
        int n = 0;
        CUDA_CHECK( cudaGetDeviceCount( &n ) );
        if( n <= 0 )
            fatal( "No CUDA device available: the B200 libssa build has no CPU path." );
        CUDA_CHECK( cudaSetDevice( dev ) );
        cudaDeviceProp prop;
        CUDA_CHECK( cudaGetDeviceProperties( &prop, dev ) );
        if( prop.major < 10 )
            fatal( "libssa B200 build needs an sm_100 device, found %s (sm_%d%d).", prop.name, prop.major,
                    prop.minor );
        sms_ = prop.multiProcessorCount;
        device_memory_ = prop.totalGlobalMem;
        CUDA_CHECK( cudaStreamCreateWithFlags( &stream_, cudaStreamNonBlocking ) );
        CUDA_CHECK( cudaEventCreate( &ev0_ ) );
        CUDA_CHECK( cudaEventCreate( &ev1_ ) );
        CUDA_CHECK( cudaEventCreateWithFlags( &ev_ready_, cudaEventDisableTiming ) );
        for( auto & e : ev_phase_ )
            CUDA_CHECK( cudaEventCreate( &e ) );
        for( auto & e : ev_seg_ )
            CUDA_CHECK( cudaEventCreate( &e ) );
        for( auto & e : ev_tb_ )
            CUDA_CHECK( cudaEventCreate( &e ) );
        for( int i = 0; i < 4; i++ ) {
            CUDA_CHECK( cudaStreamCreateWithFlags( &class_stream_[i], cudaStreamNonBlocking ) );
            CUDA_CHECK( cudaEventCreateWithFlags( &ev_class_[i], cudaEventDisableTiming ) );
            CUDA_CHECK( cudaEventCreate( &ev_cls_t_[2 * i] ) );
            CUDA_CHECK( cudaEventCreate( &ev_cls_t_[2 * i + 1] ) );
        }
        device_ = dev;
        ready_ = true;
    }

    // ---- database ------------------------------------------------------------
    const HostDb & database() {
        const Config & cfg = config();
        if( db_.symtype != cfg.symtype || db_.upi != units_per_record( cfg.symtype, cfg.strands ) || db_stale_ )
            pack_database();
        return db_;
    }

    void invalidate() { db_stale_ = true; }

    void pack_database() {
        const Config & cfg = config();
        HostDb db;
        const size_t n_rec = ssa_db_get_sequence_count();
        const uint32_t upi = units_per_record( cfg.symtype, cfg.strands );
        if( (uint64_t) n_rec * upi > UINT32_MAX )
            fatal( "Database has %zu sequences; at most %u are supported.", n_rec, UINT32_MAX / upi );
        const size_t n = n_rec * upi;
        db.n_records = (uint32_t) n_rec;
        db.upi = upi;
        db.n_ids = (uint32_t) n;
        db.len.assign( n, 0 );
        db.off.assign( n, 0 );
        const bool nt = cfg.symtype == NUCLEOTIDE;
        if( cfg.symtype == TRANS_DB || cfg.symtype == TRANS_BOTH )
            fatal( "Searches of a translated database (symbol type %d) are not supported by the B200 build.",
                    cfg.symtype );
        std::vector<p_seqinfo> infos( n_rec );
        for( size_t id = 0; id < n_rec; id++ ) {
            p_seqinfo info = ssa_db_get_sequence( id );
            if( !info )
                fatal( "Could not get sequence from DB: %zu", id );
            infos[id] = info;
            if( info->seqlen > (size_t) INT32_MAX / 2 )
                fatal( "Database sequence %zu is too long (%zu residues).", id, info->seqlen );
            for( uint32_t k = 0; k < upi; k++ )
                db.len[id * upi + k] = (uint32_t) info->seqlen;
            db.max_len = std::max( db.max_len, (uint32_t) info->seqlen );
            db.residues += (uint64_t) info->seqlen * upi;
        }
        db.nonempty_before.assign( (size_t) n + 1, 0 );
        for( uint32_t id = 0; id < db.n_ids; id++ ) {
            db.nonempty_before[id + 1] = db.nonempty_before[id] + (db.len[id] ? 1 : 0);
            if( db.len[id] )
                db.order_desc.push_back( id );
        }
        std::stable_sort( db.order_desc.begin(), db.order_desc.end(),
                [&]( uint32_t a, uint32_t b ) { return db.len[a] > db.len[b]; } );
        auto padded = [&]( uint32_t id ) { return ((uint64_t) db.len[id] + 15) & ~(uint64_t) 15; };

        // Resident layout: every ID in ID order, plus the interleaved pairs of
        // the single-query pass.  Streaming layout (the resident one does not
        // fit the database memory): segments of consecutive IDs in length
        // order, each a contiguous block that is copied to the device when its
        // turn comes; the device offsets are relative to the block.
        init_device();
        uint64_t codes_bytes = 0;
        for( uint32_t id = 0; id < db.n_ids; id++ )
            codes_bytes += padded( id );
        const uint64_t resident_bytes = 2 * codes_bytes + (uint64_t) n * (8 + 4 + 4) + 64;
        const uint64_t budget = db_budget();
        streaming_ = resident_bytes > budget;
        seg_lo_.clear();
        seg_hi_.clear();
        seg_off_.clear();
        seg_bytes_.clear();
        std::vector<uint64_t> dev_off( n, 0 );
        uint64_t total = 0;
        if( !streaming_ ) {
            for( uint32_t id = 0; id < db.n_ids; id++ ) {
                db.off[id] = total;
                dev_off[id] = total;
                total += padded( id );
            }
        }
        else {
            const uint64_t seg_cap = std::max<uint64_t>( 1, budget / 2 );
            uint64_t in_seg = 0;
            for( uint32_t pos = 0; pos < (uint32_t) db.order_desc.size(); pos++ ) {
                const uint32_t id = db.order_desc[pos];
                if( seg_lo_.empty() || (in_seg > 0 && in_seg + padded( id ) > seg_cap) ) {
                    if( !seg_lo_.empty() ) {
                        seg_hi_.push_back( pos );
                        seg_bytes_.push_back( in_seg );
                    }
                    seg_lo_.push_back( pos );
                    seg_off_.push_back( total );
                    in_seg = 0;
                }
                db.off[id] = total;
                dev_off[id] = in_seg;
                total += padded( id );
                in_seg += padded( id );
            }
            if( !seg_lo_.empty() ) {
                seg_hi_.push_back( (uint32_t) db.order_desc.size() );
                seg_bytes_.push_back( in_seg );
            }
        }
        db.codes.assign( total + 16, 0 );
        uint64_t unknown = 0;
        for( size_t id = 0; id < n_rec; id++ ) {
            // unknown symbols become code 0 (reference: src/util/util_sequence.c:298-318)
            const char * s = infos[id]->seq;
            const size_t L = infos[id]->seqlen;
            if( L == 0 )
                continue;
            uint8_t * o = db.codes.data() + db.off[id * upi];
            for( size_t k = 0; k < L; k++ ) {
                int m = nt ? map_nt16( (unsigned char) s[k] ) : map_aa( (unsigned char) s[k] );
                if( m < 0 ) {
                    m = 0;
                    unknown++;
                }
                o[k] = (uint8_t) m;
            }
            if( upi == 2 ) {
                // the reverse complement unit (reference: src/util/util_sequence.c:420-437)
                uint8_t * rc = db.codes.data() + db.off[id * upi + 1];
                for( size_t k = 0; k < L; k++ )
                    rc[k] = nt_complement( o[L - 1 - k] );
            }
        }
        if( unknown )
            print_warning( "%llu unknown symbols found and set to zero", (unsigned long long) unknown );
        db.symtype = cfg.symtype;
        db.strands = cfg.strands;
        db.generation = ++generation_;
        db.mean_len = db.order_desc.empty() ? 0.0 : (double) db.residues / (double) db.order_desc.size();

        d_off_.ensure( sizeof(uint64_t) * std::max<size_t>( 1, n ) );
        d_len_.ensure( sizeof(uint32_t) * std::max<size_t>( 1, n ) );
        d_order_.ensure( sizeof(uint32_t) * std::max<size_t>( 1, db.order_desc.size() ) );
        if( n ) {
            CUDA_CHECK( cudaMemcpy( d_off_.p, dev_off.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice ) );
            CUDA_CHECK( cudaMemcpy( d_len_.p, db.len.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice ) );
        }
        if( !db.order_desc.empty() )
            CUDA_CHECK( cudaMemcpy( d_order_.p, db.order_desc.data(), sizeof(uint32_t) * db.order_desc.size(),
                    cudaMemcpyHostToDevice ) );
        resident_seg_ = -1;
        if( streaming_ ) {
            DevBuf * big[] = { &d_codes_, &d_pair_res_, &d_pair_off_, &d_pair_cols_, &d_pair_ids_ };
            for( DevBuf * b : big )
                b->release();
            uint64_t max_seg = 0;
            for( uint64_t b : seg_bytes_ )
                max_seg = std::max( max_seg, b );
            for( DevBuf & b : d_seg_ )
                b.ensure( max_seg + 64 );
            db_ = std::move( db );
            db_stale_ = false;
            ranks_.clear();
            return;
        }
        for( DevBuf & b : d_seg_ )
            b.release();

        // pairs of consecutive sequences in length order share the 16x2 lanes
        // of the fast Smith-Waterman pass; columns past a sequence's last
        // 4-column block hold the neutral pad code
        const size_t n_pairs = (db.order_desc.size() + 1) / 2;
        db.pair_cols.resize( n_pairs );
        db.pair_a.resize( n_pairs );
        db.pair_b.resize( n_pairs );
        std::vector<uint64_t> pair_off( n_pairs + 1, 0 );
        for( size_t pi = 0; pi < n_pairs; pi++ ) {
            db.pair_a[pi] = db.order_desc[2 * pi];
            db.pair_b[pi] = (2 * pi + 1 < db.order_desc.size()) ? db.order_desc[2 * pi + 1] : 0xffffffffu;
            db.pair_cols[pi] = (db.len[db.pair_a[pi]] + 7u) & ~7u;
            pair_off[pi + 1] = pair_off[pi] + 2ull * db.pair_cols[pi];
        }
        std::vector<uint8_t> pair_res( pair_off[n_pairs] + 16, (uint8_t) FAST_PAD_CODE );
        for( size_t pi = 0; pi < n_pairs; pi++ ) {
            uint8_t * out = pair_res.data() + pair_off[pi];
            for( int half = 0; half < 2; half++ ) {
                const uint32_t id = half ? db.pair_b[pi] : db.pair_a[pi];
                if( id == 0xffffffffu )
                    continue;
                const uint32_t L = db.len[id], Lb = (L + 3u) & ~3u;
                const uint8_t * src = db.codes.data() + db.off[id];
                for( uint32_t j = 0; j < L; j++ )
                    out[2 * j + half] = src[j];
                for( uint32_t j = L; j < Lb; j++ )
                    out[2 * j + half] = 0;   // the reference's pad inside the last block
            }
        }
        d_codes_.ensure( db.codes.size() );
        CUDA_CHECK( cudaMemcpy( d_codes_.p, db.codes.data(), db.codes.size(), cudaMemcpyHostToDevice ) );
        {
            std::vector<uint2> ids( std::max<size_t>( 1, n_pairs ) );
            for( size_t pi = 0; pi < n_pairs; pi++ )
                ids[pi] = make_uint2( db.pair_a[pi], db.pair_b[pi] );
            d_pair_res_.ensure( pair_res.size() );
            d_pair_off_.ensure( sizeof(uint64_t) * (n_pairs + 1) );
            d_pair_cols_.ensure( sizeof(uint32_t) * std::max<size_t>( 1, n_pairs ) );
            d_pair_ids_.ensure( sizeof(uint2) * ids.size() );
            CUDA_CHECK( cudaMemcpy( d_pair_res_.p, pair_res.data(), pair_res.size(), cudaMemcpyHostToDevice ) );
            CUDA_CHECK( cudaMemcpy( d_pair_off_.p, pair_off.data(), sizeof(uint64_t) * (n_pairs + 1),
                    cudaMemcpyHostToDevice ) );
            if( n_pairs )
                CUDA_CHECK( cudaMemcpy( d_pair_cols_.p, db.pair_cols.data(), sizeof(uint32_t) * n_pairs,
                        cudaMemcpyHostToDevice ) );
            CUDA_CHECK( cudaMemcpy( d_pair_ids_.p, ids.data(), sizeof(uint2) * ids.size(), cudaMemcpyHostToDevice ) );
        }
        db_ = std::move( db );
        db_stale_ = false;
        ranks_.clear();
    }

    DbView db_view() const {
        DbView v;
        v.codes = streaming_ ? d_seg_[resident_seg_ & 1].as<uint8_t>() : d_codes_.as<uint8_t>();
        v.offsets = d_off_.as<uint64_t>();
        v.lens = d_len_.as<uint32_t>();
        v.n_ids = db_.n_ids;
        return v;
    }

    const uint32_t * ranks( size_t chunk_size, int lanes ) {
        for( auto & c : ranks_ )
            if( c.chunk_size == chunk_size && c.lanes == lanes && c.generation == db_.generation )
                return c.rank.data();
        ScheduleCache c;
        c.chunk_size = chunk_size;
        c.lanes = lanes;
        c.generation = db_.generation;
        schedule_ranks( db_, chunk_size, lanes, c.rank );
        ranks_.push_back( std::move( c ) );
        return ranks_.back().rank.data();
    }

    // ---- search ----------------------------------------------------------------
    void search( const SearchRequest & req, const std::vector<QueryCodes> & queries,
            const std::vector<uint32_t> & groups, std::vector<std::vector<Hit>> & out, SearchStats & stats );
    // query i against database unit units[i] alone
    void align_pairs( const SearchRequest & req, const std::vector<QueryCodes> & queries,
            const std::vector<uint32_t> & units, std::vector<std::vector<Hit>> & out, SearchStats & stats );
    // database-sharded search: entry pass and cascade of every query against
    // the records [id_lo, id_hi) only; per (query, record) the final score and
    // the blocks the entry-width and 16-bit lanes spent when they overflowed
    void shard_scores( const SearchRequest & req, const std::vector<QueryCodes> & queries, uint32_t id_lo,
            uint32_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16, SearchStats & stats );
    // traceback of replayed hit lists (out[q] for query q)
    void align_hits( const SearchRequest & req, const std::vector<QueryCodes> & queries,
            std::vector<std::vector<Hit>> & out, SearchStats & stats );
    void set_traceback_budget( uint64_t bytes ) { tb_budget_ = bytes; }
    void set_db_budget( uint64_t bytes ) {
        db_budget_ = bytes;
        db_stale_ = true;
    }
    bool streaming() const { return streaming_; }

    // Device memory for the database: the setting of ssa_b200_set_db_memory,
    // else 40% of the device memory (scores, re-queue lists, profiles and
    // traceback matrices take the rest).
    uint64_t db_budget() {
        if( db_budget_ )
            return db_budget_;
        size_t free_b = 0, total_b = 0;
        CUDA_CHECK( cudaMemGetInfo( &free_b, &total_b ) );
        return (uint64_t) total_b / 5 * 2;
    }

    // Segment s of a streamed database on the device (the other buffer keeps
    // the previous one); a no-op when it is there already.
    void make_resident( uint32_t sg, SearchStats & stats ) {
        if( !streaming_ || resident_seg_ == (int) sg )
            return;
        const uint64_t bytes = seg_bytes_[sg];
        uint8_t * stage = (uint8_t *) h_stage_.ensure( std::max<uint64_t>( bytes, 16 ) );
        // the staging buffer is reused: the previous copy must have finished
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        memcpy( stage, db_.codes.data() + seg_off_[sg], bytes );
        CUDA_CHECK( cudaMemcpyAsync( d_seg_[sg & 1].p, stage, bytes, cudaMemcpyHostToDevice, stream_ ) );
        resident_seg_ = (int) sg;
        stats.h2d_bytes += bytes;
    }

    // A device view of the given database IDs alone (in that order, view ID k =
    // ids[k]), for passes over a few sequences of a streamed database.
    DbView gather_view( const std::vector<uint32_t> & ids, SearchStats & stats ) {
        std::vector<uint64_t> off( ids.size() + 1, 0 );
        std::vector<uint32_t> len( std::max<size_t>( 1, ids.size() ), 0 );
        for( size_t k = 0; k < ids.size(); k++ ) {
            len[k] = db_.len[ids[k]];
            off[k + 1] = off[k] + (((uint64_t) len[k] + 15) & ~(uint64_t) 15);
        }
        std::vector<uint8_t> codes( off[ids.size()] + 64, 0 );
        for( size_t k = 0; k < ids.size(); k++ )
            memcpy( codes.data() + off[k], db_.codes.data() + db_.off[ids[k]], len[k] );
        d_gather_codes_.ensure( codes.size() );
        d_gather_off_.ensure( off.size() * sizeof(uint64_t) );
        d_gather_len_.ensure( len.size() * sizeof(uint32_t) );
        CUDA_CHECK( cudaMemcpyAsync( d_gather_codes_.p, codes.data(), codes.size(), cudaMemcpyHostToDevice, stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( d_gather_off_.p, off.data(), off.size() * sizeof(uint64_t),
                cudaMemcpyHostToDevice, stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( d_gather_len_.p, len.data(), len.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice, stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );   // the host vectors go out of scope
        stats.h2d_bytes += codes.size() + off.size() * sizeof(uint64_t) + len.size() * sizeof(uint32_t);
        DbView v;
        v.codes = d_gather_codes_.as<uint8_t>();
        v.offsets = d_gather_off_.as<uint64_t>();
        v.lens = d_gather_len_.as<uint32_t>();
        v.n_ids = (uint32_t) ids.size();
        return v;
    }

    void shutdown() {
        DevBuf * bufs[] = { &d_codes_, &d_off_, &d_len_, &d_order_, &d_pair_res_, &d_pair_off_, &d_pair_cols_,
            &d_pair_ids_, &d_prof8_, &d_prof8_off_, &d_rows_, &d_slots_, &d_bounds_, &d_group_,
            &d_scratch_fast_[0], &d_scratch_fast_[1], &d_scratch_fast_[2], &d_scratch_fast_[3], &d_scratch_fast_[4],
            &d_scratch_fast_[5], &d_scratch_fast_[6], &d_scratch_fast_[7], &d_qcodes_, &d_qoff_, &d_qlen_, &d_qpad_,
            &d_prof_off_, &d_prof_, &d_matrix_, &d_score_, &d_list_a_, &d_list_b_, &d_counts_, &d_scratch_,
            &d_tb_hits_, &d_tb_regions_, &d_tb_last_, &d_tb_last_off_, &d_tb_dirs_, &d_tb_dir_off_, &d_tb_ops_,
            &d_tb_ops_off_, &d_tb_ops_len_, &d_qp_prof_, &d_qp_off_, &d_qp_rows_, &d_qp_slots_, &d_qp_units_,
            &d_serve_score_, &d_qp_lmax_, &d_pair_slot_, &d_pair_unit_, &d_pair_score_, &d_scratch2_, &d_scratch4_,
            &d_seg_[0], &d_seg_[1], &d_gather_codes_, &d_gather_off_, &d_gather_len_, &d_prof64_, &d_score64_ };
        for( DevBuf * b : bufs )
            b->release();
        h_score_.release();
        h_score64_.release();
        h_stage_.release();
        resident_seg_ = -1;
        streaming_ = false;
        db_ = HostDb();
        db_stale_ = true;
        ranks_.clear();
        serve_layout_ = false;
        serve_slots_ = 0;
        serve_codes_.clear();
    }

    uint64_t launches() const { return launches_.load(); }

    // ---- serving: fixed query slots, waves over database segments ---------------
    std::vector<uint32_t> serve_open( const SearchRequest & req, uint32_t slots, uint32_t segments );
    void serve_restore( const SearchRequest & req );
    void serve_load( uint32_t slot, const uint8_t * codes, uint32_t len );
    void serve_wave( const SearchRequest & req, const std::vector<uint32_t> & active, uint32_t seq_lo,
            uint32_t seq_hi, std::vector<PairTask> & ovf_entry, std::vector<PairTask> & ovf16, SearchStats & stats );
    void serve_finish( const SearchRequest & req, const std::vector<uint32_t> & done,
            std::vector<ReplayQuery> & rq, std::vector<std::vector<Hit>> & out, SearchStats & stats );

private:
    Engine() = default;

    void run_pass( int algo, int width, const SearchRequest & req, uint32_t n_slots, const PairTask * tasks,
            uint64_t n_tasks, bool implicit, PairTask * next, unsigned * next_count, uint32_t next_cap,
            const uint32_t * slot_list = nullptr, uint32_t n_sub = 0, uint32_t order_lo = 0 );
    void run_fast_entry( const SearchRequest & req, uint32_t nq, PairTask * next, unsigned * next_count, uint32_t cap );
    void run_qpair_entry( const SearchRequest & req, uint32_t nq, PairTask * next, unsigned * next_count,
            uint32_t cap, const std::vector<uint32_t> * slots = nullptr, uint32_t seq_lo = 0,
            uint32_t seq_hi = UINT32_MAX );
    int32_t * score_sink() { return serving_ ? d_serve_score_.as<int32_t>() : d_score_.as<int32_t>(); }
    void build_profiles( int width, uint32_t n_slots );
    // scores_from_regions: the hits carry no score yet; take it from the
    // forward pass (SW, symmetric table) or the direction pass (NW)
    void traceback( const SearchRequest & req, std::vector<std::vector<Hit>> & out,
            const std::vector<std::pair<uint32_t, uint32_t>> & lists, SearchStats & stats,
            bool scores_from_regions = false );
    uint64_t traceback_budget();
    void upload_queries( const QueryCodes * queries, uint32_t nq, bool profiles, SearchStats & stats );

    bool ready_ = false;
    int device_ = 0;
    int sms_ = 148;
    uint64_t device_memory_ = 0;
    // (query, sequence) pairs of one sub-batch: its int32 scores (4 B) and, at
    // most, two re-queue lists of 16 B per pair; 2^29 pairs (19 GB) on devices
    // of 64 GB and more (a 1,024-query batch against 500,000 sequences in one
    // pass), 2^28 otherwise; halved when the 64-bit pass keeps int64 scores
    uint64_t pair_budget() const {
        const int log2 = device_memory_ >= ((uint64_t) 64 << 30) ? 29 : 28;
        return (uint64_t) 1 << (wide_ ? log2 - 1 : log2);
    }
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    HostDb db_;
    bool db_stale_ = true;
    uint64_t generation_ = 0;
    std::vector<ScheduleCache> ranks_;
    std::atomic<uint64_t> launches_{ 0 };

    // device buffers
    DevBuf d_codes_, d_off_, d_len_, d_order_;
    DevBuf d_pair_res_, d_pair_off_, d_pair_cols_, d_pair_ids_;
    DevBuf d_prof8_, d_prof8_off_, d_rows_, d_slots_;
    DevBuf d_scratch_fast_[8];      // per class of the single-query pass
    DevBuf d_bounds_, d_group_;
    DevBuf d_qp_prof_, d_qp_off_, d_qp_rows_, d_qp_slots_, d_qp_units_, d_qp_lmax_;
    // serving: fixed query slots and their own score rows
    DevBuf d_serve_score_;
    bool serving_ = false;           // passes write d_serve_score_
    bool serve_layout_ = false;      // the query buffers hold the serving slots
    uint32_t serve_slots_ = 0;
    std::vector<std::vector<uint8_t>> serve_codes_;   // per slot, to restore the layout after a search
    cudaStream_t class_stream_[4] = { nullptr, nullptr, nullptr, nullptr };
    cudaEvent_t ev_class_[4] = { nullptr, nullptr, nullptr, nullptr };
    cudaEvent_t ev_cls_t_[8] = {};   // per class start / end, timed (SSA_B200_TIMING)
    cudaEvent_t ev_ready_ = nullptr;
    cudaEvent_t ev_phase_[6] = {};
    cudaEvent_t ev_seg_[2] = {};     // around one segment's entry pass
    cudaEvent_t ev_tb_[5] = {};   // batch start, entry pass done, cascade done, copies done, traceback
    DevBuf d_qcodes_, d_qoff_, d_qlen_, d_qpad_, d_prof_off_, d_prof_, d_matrix_;
    DevBuf d_score_, d_list_a_, d_list_b_, d_counts_, d_scratch_, d_scratch2_, d_scratch4_;
    DevBuf d_tb_hits_, d_tb_regions_, d_tb_last_, d_tb_last_off_, d_tb_dirs_, d_tb_dir_off_, d_tb_ops_,
            d_tb_ops_off_, d_tb_ops_len_;
    PinnedBuf h_score_;
public:
    // entry-pass shapes of the last search call: kernel, (R, CTAs per SM) for
    // the query-pair kernel or (G, R) for the single-query one, queries or
    // query pairs, database bucket
    struct ShapeUse {
        const char * kernel;
        int a, b;
        uint32_t n;
        int bucket;
    };
    std::vector<ShapeUse> last_shapes_;
private:
    // the 64-bit pass in int64 arithmetic (wide_): exact profiles and scores
    DevBuf d_prof64_, d_score64_;
    PinnedBuf h_score64_;
    bool wide_ = false;
    int prof64_width_ = -1;
    DevBuf d_pair_slot_, d_pair_unit_, d_pair_score_;
    uint64_t tb_budget_ = 0;         // traceback direction memory per wave (0 = automatic)
    // streaming: the database does not fit its device memory budget; segments
    // of consecutive positions of the length order take turns on the device
    uint64_t db_budget_ = 0;         // database device memory (0 = automatic)
    bool streaming_ = false;
    std::vector<uint32_t> seg_lo_, seg_hi_;     // per segment: positions in order_desc
    std::vector<uint64_t> seg_off_, seg_bytes_; // per segment: block in db_.codes
    DevBuf d_seg_[2];
    int resident_seg_ = -1;
    PinnedBuf h_stage_;
    DevBuf d_gather_codes_, d_gather_off_, d_gather_len_;

    // per-batch query layout
    std::vector<uint64_t> h_qoff_;
    std::vector<uint32_t> h_qlen_, h_qpad_;
    std::vector<uint64_t> h_prof_off_;
    int prof_width_ = -1;
    uint32_t prof_slots_ = 0;
    uint32_t max_qlen_ = 0;

    friend void engine_shutdown();
};

void Engine::build_profiles( int width, uint32_t n_slots ) {
    if( wide_ && width == 64 ) {
        // exact int64 table (same offsets as the int32 one, twice the bytes)
        if( prof_width_ == 64 && prof64_width_ == 64 && prof_slots_ == n_slots )
            return;
        uint64_t elems = 0;
        for( uint32_t s = 0; s < n_slots && s < h_prof_off_.size(); s++ )
            elems = std::max<uint64_t>( elems, h_prof_off_[s] + 32ull * h_qpad_[s] );
        d_prof64_.ensure( std::max<uint64_t>( elems, 1 ) * sizeof(int64_t) );
        CUDA_CHECK( launch_build_profile64( d_qcodes_.as<uint8_t>(), d_qoff_.as<uint64_t>(), d_qlen_.as<uint32_t>(),
                d_qpad_.as<uint32_t>(), d_prof_off_.as<uint64_t>(), d_matrix_.as<int64_t>(), d_prof64_.as<int64_t>(),
                n_slots, stream_ ) );
        launches_++;
        prof_width_ = 64;
        prof64_width_ = 64;
        prof_slots_ = n_slots;
        return;
    }
    if( prof_width_ == width && prof_slots_ == n_slots && prof64_width_ != 64 )
        return;
    launch_build_profile32( d_qcodes_.as<uint8_t>(), d_qoff_.as<uint64_t>(), d_qlen_.as<uint32_t>(),
            d_qpad_.as<uint32_t>(), d_prof_off_.as<uint64_t>(), d_matrix_.as<int64_t>(), width,
            d_prof_.as<int32_t>(), n_slots, stream_ );
    CUDA_CHECK( cudaGetLastError() );
    launches_++;
    prof_width_ = width;
    prof64_width_ = -1;
    prof_slots_ = n_slots;
}

void Engine::run_pass( int algo, int width, const SearchRequest & req, uint32_t n_slots, const PairTask * tasks,
        uint64_t n_tasks, bool implicit, PairTask * next, unsigned * next_count, uint32_t next_cap,
        const uint32_t * slot_list, uint32_t n_sub, uint32_t order_lo ) {
    if( n_tasks == 0 )
        return;
    build_profiles( width, n_slots );
    EmulParams p;
    p.db = db_view();
    p.qv.prof32 = d_prof_.as<int32_t>();
    p.qv.prof32_off = d_prof_off_.as<uint64_t>();
    p.qv.qlen = d_qlen_.as<uint32_t>();
    p.qv.qpad = d_qpad_.as<uint32_t>();
    p.qv.n_slots = n_slots;
    p.tasks = implicit ? nullptr : tasks;
    p.order = d_order_.as<uint32_t>() + order_lo;
    p.slot_list = slot_list;
    p.n_sub = n_sub;
    p.n_tasks = n_tasks;
    unsigned long long * counter = d_counts_.as<unsigned long long>() + 4;
    CUDA_CHECK( cudaMemsetAsync( counter, 0, sizeof(unsigned long long), stream_ ) );
    p.counter = counter;
    p.gap_open = req.gap_open;
    p.gap_extend = req.gap_extend;
    p.sink.score = score_sink();
    p.sink.score_stride = db_.n_ids;
    p.sink.next = next;
    p.sink.next_count = next_count;
    p.sink.next_cap = next_cap;
    p.sink.error_flags = d_counts_.as<unsigned>() + 2;
    const bool wide = wide_ && width == 64;
    if( wide ) {
        if( serving_ )
            fatal( "Internal error: int64 scoring is not available to the server." );
        p.qv.prof64 = d_prof64_.as<int64_t>();
        p.sink.score64 = d_score64_.as<int64_t>();
    }
    const int grid = sms_ * 2;
    const uint32_t cols = ((db_.max_len + 3u) & ~3u) + 4;
    if( max_qlen_ > 256 ) {
        // a boundary column is 4 values: 16 bytes in int32, 32 in int64
        const size_t col_bytes = wide ? 2 * sizeof(int4) : sizeof(int4);
        p.scratch = (int4 *) d_scratch_.ensure( (size_t) grid * 8 * cols * col_bytes );
        p.scratch_cols = cols;
    }
    else {
        p.scratch = nullptr;
        p.scratch_cols = 0;
    }
    CUDA_CHECK( launch_emul( algo, width, p, grid, stream_, wide ) );
    launches_++;
}

// Whether the 64-bit pass needs int64 arithmetic: a DP value is bounded by the
// number of steps of a path (query rows + columns + a few boundary terms) times
// the largest magnitude of one step (a score-table entry, or gapO + gapE); at
// or below the int32 range (with a factor 2 of margin for the sums formed
// before each max) int32 is exact.
static bool needs_int64( const SearchRequest & req, uint32_t max_qlen, uint32_t max_dlen ) {
    int64_t m = std::llabs( (int64_t) req.gap_open ) + std::llabs( (int64_t) req.gap_extend );
    for( int k = 0; k < 1024; k++ )
        m = std::max<int64_t>( m, req.matrix[k] == INT64_MIN ? INT64_MAX / 4 : std::llabs( req.matrix[k] ) );
    const int64_t steps = (int64_t) max_qlen + max_dlen + 8;
    return m > (int64_t) INT32_MAX / 2 || steps * (m + 1) * 2 > (int64_t) INT32_MAX;
}

// The 16x2 pass reproduces the 8-bit Smith-Waterman lanes exactly when the
// gap extension is not positive and the truncated 8-bit open+extend cost lies
// in [-128, gapE]; other parameters run the exact lane emulation.
// Needleman-Wunsch at the 16-bit entry: the query-pair kernel scores exactly
// the sequences short enough that no value can come near the int16 limits
// (nw_qpair_kernel); it needs non-positive gap costs.
static bool nw_fast_eligible( const SearchRequest & req ) {
    if( req.algo != 1 || req.bit_width != 16 || getenv( "SSA_B200_NO_FAST" ) )
        return false;
    return req.gap_open <= 0 && req.gap_extend <= 0;
}

static bool fast_eligible( const SearchRequest & req ) {
    if( req.algo != 0 || req.bit_width != 8 )
        return false;
    if( getenv( "SSA_B200_NO_FAST" ) )
        return false;
    // the kernel also uses gapO + gapE <= gapE (in 8-bit terms) to let the next
    // row's F depend on Hdiag + V and E only
    const int goe8 = (int8_t) (req.gap_open + req.gap_extend);
    return req.gap_extend <= 0 && goe8 <= 0 && goe8 <= req.gap_extend;
}

struct FastShape {
    int G, R, P;
    int C;      // columns per step: 1 (sw_fast_kernel) or 4 (sw_fast4_kernel)
};

constexpr uint32_t FAST_MAX_ROWS = 8192;    // longer queries run the lane emulation
constexpr uint32_t FAST_MAX_PASS_ROWS = 512; // G x R: 16 KiB profile slice per warp

// Threads per group G, rows per thread R, passes P and columns per step C for
// a query of Q rows: without a measured table, the one-column kernel with the
// smallest estimated issue cost per database column, counting the wavefront
// fill (G - 1 steps per pass) and a per-step overhead.  With a measured shape
// table for the database's bucket (tuning.cpp) the cost of a shape is
// passes x its measured cost per pass and column, over both kernels; on a
// small database that measurement includes the latency of the longest pairs,
// so it favours wide groups there.
static FastShape choose_shape( uint32_t Q, double mean_len, int bucket ) {
    FastShape best{ 0, 0, 0, 1 };
    double best_cost = 1e300;
    const int Gs[] = { 8, 16, 32 };
    const int G4s[] = { 4, 8, 16, 32 };
    const int Rs[] = { 8, 16, 24, 32 };
    const TuningTable & tt = tuning();
    bool measured = false, measured4 = false;
    for( int gi = 0; gi < 3 && tt.has_fast; gi++ )
        for( int ri = 0; ri < 4; ri++ )
            measured |= tt.fast[bucket][gi][ri] > 0;
    for( int gi = 0; gi < 4 && tt.has_fast4; gi++ )
        for( int ri = 0; ri < 4; ri++ )
            measured4 |= tt.fast4[bucket][gi][ri] > 0;
    auto fits = []( int G, int R, uint32_t Q, uint32_t * P ) {
        const uint32_t per = (uint32_t) (G * R);
        *P = (Q + per - 1) / per;
        return per <= FAST_MAX_PASS_ROWS && (uint64_t) *P * per <= FAST_MAX_ROWS;
    };
    // the model's cost units are not the table's: with only the 4-column
    // kernel measured, the one-column kernel is not a candidate
    if( measured || !measured4 ) {
        for( int gi = 0; gi < 3; gi++ ) {
            const int G = Gs[gi];
            for( int ri = 0; ri < 4; ri++ ) {
                const int R = Rs[ri];
                uint32_t P;
                if( !fits( G, R, Q, &P ) )
                    continue;
                if( measured && tt.fast[bucket][gi][ri] <= 0 )
                    continue;
                const double cost = measured ? (double) P * tt.fast[bucket][gi][ri]
                                             : (double) P * G * (mean_len + G - 1) * (8.0 * R + 24.0);
                if( cost < best_cost ) {
                    best_cost = cost;
                    best = FastShape{ G, R, (int) P, 1 };
                }
            }
        }
    }
    for( int gi = 0; gi < 4 && measured4; gi++ ) {
        const int G = G4s[gi];
        for( int ri = 0; ri < 3; ri++ ) {     // R = 8, 16, 24
            const int R = Rs[ri];
            uint32_t P;
            if( !fits( G, R, Q, &P ) || tt.fast4[bucket][gi][ri] <= 0 )
                continue;
            const double cost = (double) P * tt.fast4[bucket][gi][ri];
            if( cost < best_cost ) {
                best_cost = cost;
                best = FastShape{ G, R, (int) P, 4 };
            }
        }
    }
    return best;
}

void Engine::run_fast_entry( const SearchRequest & req, uint32_t nq, PairTask * next, unsigned * next_count,
        uint32_t cap ) {
    const uint32_t n_pairs = (uint32_t) db_.pair_cols.size();
    if( n_pairs == 0 )
        return;
    // shape per slot; queries too long for the shared-memory profile run the
    // exact lane emulation instead
    std::vector<FastShape> shape( nq );
    std::vector<uint32_t> rows_of( nq, 0 );
    std::vector<uint32_t> fallback;
    // classes: [columns per step 1 or 4][R = 8, 16, 24, 32]
    std::vector<std::vector<uint32_t>> by_r( 8 );
    const int bucket = db_bucket( db_.mean_len, db_.order_desc.size() );
    // SSA_B200_FAST_SHAPE=G,R[,C] pins the shape and the kernel (tuning, tests)
    int pin_g = 0, pin_r = 0, pin_c = 1;
    if( const char * pin = getenv( "SSA_B200_FAST_SHAPE" ) ) {
        const int n = sscanf( pin, "%d,%d,%d", &pin_g, &pin_r, &pin_c );
        const bool g_ok = pin_c == 4 ? (pin_g == 4 || pin_g == 8 || pin_g == 16 || pin_g == 32)
                                     : (pin_g == 8 || pin_g == 16 || pin_g == 32);
        const int r_max = pin_c == 4 ? 24 : 32;
        if( n < 2 || (n == 3 && pin_c != 1 && pin_c != 4) || !g_ok || pin_r < 8 || pin_r > r_max || pin_r % 8 )
            pin_g = pin_r = 0;
    }
    for( uint32_t s = 0; s < nq; s++ ) {
        shape[s] = choose_shape( h_qlen_[s], db_.mean_len, bucket );
        if( pin_g && shape[s].G ) {
            const uint32_t per = (uint32_t) (pin_g * pin_r);
            const uint32_t P = (h_qlen_[s] + per - 1) / per;
            if( per <= FAST_MAX_PASS_ROWS && (uint64_t) P * per <= FAST_MAX_ROWS )
                shape[s] = FastShape{ pin_g, pin_r, (int) P, pin_c };
        }
        if( shape[s].G == 0 ) {
            fallback.push_back( s );
            continue;
        }
        rows_of[s] = (uint32_t) (shape[s].G * shape[s].R * shape[s].P);
        by_r[(shape[s].C == 4 ? 4 : 0) + shape[s].R / 8 - 1].push_back( s );
    }
    // profiles: one 32 x rows int8 table per slot
    std::vector<uint64_t> prof_off( nq, 0 );
    uint64_t total = 0;
    std::vector<uint32_t> slots;
    for( auto & v : by_r )
        for( uint32_t s : v ) {
            prof_off[s] = total;
            total += 32ull * rows_of[s];
            slots.push_back( s );
        }
    const size_t n_shaped = slots.size();
    for( uint32_t s : fallback )
        slots.push_back( s );
    d_prof8_.ensure( total + 16 );
    d_prof8_off_.ensure( nq * sizeof(uint64_t) );
    d_rows_.ensure( nq * sizeof(uint32_t) );
    d_slots_.ensure( std::max<size_t>( 1, slots.size() ) * sizeof(uint32_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_prof8_off_.p, prof_off.data(), nq * sizeof(uint64_t), cudaMemcpyHostToDevice,
            stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_rows_.p, rows_of.data(), nq * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_slots_.p, slots.data(), slots.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
            stream_ ) );
    if( n_shaped ) {
        CUDA_CHECK( launch_build_profile8( d_qcodes_.as<uint8_t>(), d_qoff_.as<uint64_t>(), d_qlen_.as<uint32_t>(),
                d_slots_.as<uint32_t>(), (uint32_t) n_shaped, d_rows_.as<uint32_t>(), d_matrix_.as<int64_t>(),
                d_prof8_.as<int8_t>(), d_prof8_off_.as<uint64_t>(), stream_ ) );
        launches_++;
    }

    // work units: ranges of length-sorted pairs holding about equal numbers
    // of columns, the longest first; every query of a class gets every range.
    // A warp takes one unit at a time and runs its pairs 32 / G at a time, so
    // a unit holds at least one such round for the smallest group of the call
    // (no idle groups) and, where the columns allow, no more: on a small
    // database the longest pairs then run side by side in separate warps
    // instead of one after another in the same warp.
    uint64_t total_cols = 0;
    for( uint32_t c : db_.pair_cols )
        total_cols += c;
    int g_min = 32;
    for( uint32_t s = 0; s < nq; s++ )
        if( shape[s].G )
            g_min = std::min( g_min, shape[s].G );
    const uint32_t min_pairs = 32u / (uint32_t) g_min;
    const uint64_t want_units = (uint64_t) sms_ * 16 * 24;   // ~24 units per resident warp
    const uint64_t target = std::max<uint64_t>( 1, total_cols * std::max<size_t>( 1, n_shaped ) / want_units );
    std::vector<uint32_t> bounds{ 0 };
    {
        uint64_t acc = 0;
        uint32_t cnt = 0;
        for( uint32_t pi = 0; pi < n_pairs; pi++ ) {
            acc += db_.pair_cols[pi];
            cnt++;
            if( acc >= target && cnt >= min_pairs ) {
                bounds.push_back( pi + 1 );
                acc = 0;
                cnt = 0;
            }
        }
        if( bounds.back() != n_pairs )
            bounds.push_back( n_pairs );
    }
    const uint32_t n_chunks = (uint32_t) bounds.size() - 1;
    std::vector<uint16_t> group_of( nq, 32 );
    for( uint32_t s = 0; s < nq; s++ )
        if( shape[s].G )
            group_of[s] = (uint16_t) shape[s].G;
    d_bounds_.ensure( bounds.size() * sizeof(uint32_t) );
    d_group_.ensure( nq * sizeof(uint16_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_bounds_.p, bounds.data(), bounds.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
            stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_group_.p, group_of.data(), nq * sizeof(uint16_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaEventRecord( ev_ready_, stream_ ) );
    const uint32_t cols_max = ((db_.max_len + 7u) & ~7u) + 8;
    size_t class_first = 0;
    for( int ci = 0; ci < 8; ci++ ) {
        const std::vector<uint32_t> & cls = by_r[ci];
        if( cls.empty() )
            continue;
        const bool four = ci >= 4;
        const int ri = ci % 4;                 // classes of equal R share a stream
        const int R = 8 * (ri + 1);
        bool multi = false;
        uint32_t slice_rows = 0;
        for( uint32_t s : cls ) {
            multi |= shape[s].P > 1;
            slice_rows = std::max( slice_rows, (uint32_t) (shape[s].G * R) );
        }
        {
            std::map<int, uint32_t> by_g;
            for( uint32_t s : cls )
                by_g[shape[s].G]++;
            for( auto & kv : by_g )
                last_shapes_.push_back( { four ? "sw_fast4" : "sw_fast", kv.first, R, kv.second, bucket } );
        }
        auto launch = [&]( const FastParams & fp, int g, int * per ) {
            return four ? launch_sw_fast4( R, fp, g, class_stream_[ri], per )
                        : launch_sw_fast( R, fp, g, class_stream_[ri], per );
        };
        FastParams p{};
        p.slice_rows = slice_rows;
        int per_sm = 0;
        CUDA_CHECK( launch( p, 0, &per_sm ) );
        // SSA_B200_FAST_CTAS=n caps the resident CTAs per SM (tuning)
        if( const char * cap_env = getenv( "SSA_B200_FAST_CTAS" ) )
            per_sm = std::min( per_sm, std::max( 1, atoi( cap_env ) ) );
        const int grid = sms_ * std::max( 1, per_sm );
        CUDA_CHECK( cudaStreamWaitEvent( class_stream_[ri], ev_ready_, 0 ) );
        unsigned long long * unit_counter = d_counts_.as<unsigned long long>() + 8 + ri;   // bytes 64..95
        CUDA_CHECK( cudaMemsetAsync( unit_counter, 0, sizeof(unsigned long long), class_stream_[ri] ) );
        p.pair_res = d_pair_res_.as<uint8_t>();
        p.pair_off = d_pair_off_.as<uint64_t>();
        p.pair_cols = d_pair_cols_.as<uint32_t>();
        p.pair_ids = d_pair_ids_.as<uint2>();
        p.prof8 = d_prof8_.as<int8_t>();
        p.prof8_off = d_prof8_off_.as<uint64_t>();
        p.slot_group = d_group_.as<uint16_t>();
        p.slot_rows = d_rows_.as<uint32_t>();
        p.unit_slots = d_slots_.as<uint32_t>() + class_first;
        p.n_class = (uint32_t) cls.size();
        p.chunk_bounds = d_bounds_.as<uint32_t>();
        p.n_units = (uint64_t) n_chunks * cls.size();
        p.unit_counter = unit_counter;
        p.gap_oe = (int8_t) (req.gap_open + req.gap_extend);
        p.gap_e = req.gap_extend;
        p.sink.score = score_sink();
        p.sink.score_stride = db_.n_ids;
        p.sink.next = next;
        p.sink.next_count = next_count;
        p.sink.next_cap = cap;
        p.sink.error_flags = d_counts_.as<unsigned>() + 2;
        if( multi ) {
            // a scratch row per group: 4 groups per warp (8 in the 4-column kernel)
            p.scratch = (int4 *) d_scratch_fast_[ci].ensure( (size_t) grid * (FAST_THREADS / 32) * (four ? 8 : 4) *
                    cols_max * sizeof(int4) );
            p.scratch_cols = cols_max;
        }
        CUDA_CHECK( launch( p, grid, nullptr ) );
        launches_++;
        CUDA_CHECK( cudaEventRecord( ev_class_[ri], class_stream_[ri] ) );
        CUDA_CHECK( cudaStreamWaitEvent( stream_, ev_class_[ri], 0 ) );
        class_first += cls.size();
    }
    if( !fallback.empty() ) {
        const uint64_t n_ne = db_.order_desc.size();
        run_pass( 0, 8, req, nq, nullptr, (uint64_t) fallback.size() * n_ne, true, next, next_count, cap,
                d_slots_.as<uint32_t>() + n_shaped, (uint32_t) fallback.size() );
    }
}

// Batches: queries sorted by length are paired, the two queries of a pair
// share the 16x2 lanes (sw_qpair_kernel.cu).  Rows per thread R for a pair of
// Q rows (the longer query): the smallest estimated time per column pair,
// passes x cost(R), with QP_G x R rows per pass.  cost(R) is the measured
// device time of one pass per column pair on a B200 (relative units; 64
// queries of 375 residues against 10,000 sequences, each R pinned): R = 16
// pays for 2-way shared-memory bank conflicts inside a group, R = 28 for a
// few spilled registers.
// The costs come from the measured shape table (tuning.cpp): per pass and
// database column of a query pair, for each rows-per-thread R and resident
// CTAs per SM (4 or 5); the smallest passes x cost wins.  pinned_r / pinned_mb
// (SSA_B200_QP_R, SSA_B200_QP_MB) force a shape, as the tuner does.
struct QpVariant {
    int mb;         // resident CTAs per SM
    int cols;       // columns per step
    bool hmax;      // running maximum in fp16x2 (4 columns, 4 CTAs per SM)
    bool g8;        // 8 threads of 12 rows per sequence (R = 24, 4 columns)
    double cost;    // measured cost, 0 = none
};

// The cheapest measured variant of the query-pair kernel for rows-per-thread
// R (pinned_mb / pinned_c / pinned_h / pinned_g8 force one; pinned_h and
// pinned_g8: 0 or 1, -1 = free).
static QpVariant qpair_variant( int bucket, int R, int pinned_mb, int pinned_c, int pinned_h, int pinned_g8 ) {
    QpVariant best{ 4, 2, false, false, 0 };
    for( int mi = 0; mi < 2; mi++ )
        for( int vi = 0; vi < 4; vi++ ) {
            const int mb = 4 + mi, cols = vi ? 4 : 2;
            const bool hm = vi == 2, g8 = vi == 3;
            if( (hm && mb != 4) || (g8 && R != 24) )
                continue;
            if( (pinned_mb == 4 || pinned_mb == 5) && mb != pinned_mb )
                continue;
            if( (pinned_c == 2 || pinned_c == 4) && cols != pinned_c )
                continue;
            if( pinned_h >= 0 && hm != (pinned_h == 1) )
                continue;
            if( pinned_g8 >= 0 && g8 != (pinned_g8 == 1) )
                continue;
            const double c = tuning().qpair[bucket][R / 4 - 4][mi][vi];
            if( c > 0 && (best.cost <= 0 || c < best.cost) )
                best = QpVariant{ mb, cols, hm, g8, c };
        }
    if( best.cost <= 0 ) {
        if( pinned_mb == 4 || pinned_mb == 5 )
            best.mb = pinned_mb;
        if( pinned_c == 2 || pinned_c == 4 )
            best.cols = pinned_c;
        if( pinned_h == 1 ) {
            best.cols = 4;
            best.mb = 4;
            best.hmax = true;
        }
        else if( pinned_g8 == 1 && R == 24 ) {
            best.cols = 4;
            best.g8 = true;
        }
    }
    return best;
}

static int choose_qpair_rows( uint32_t Q, uint32_t * passes, int pinned, int bucket, int pinned_mb, int pinned_c,
        int pinned_h, int pinned_g8 ) {
    static const int rs[4] = { 16, 20, 24, 28 };
    int best_r = 0;
    double best_cost = 1e300;
    for( int i = 0; i < 4; i++ ) {
        const int R = rs[i];
        if( pinned && R != pinned )
            continue;
        const uint32_t per = (uint32_t) (QP_G * R);
        const uint32_t P = std::max<uint32_t>( 1, (Q + per - 1) / per );
        if( (uint64_t) P * per > FAST_MAX_ROWS )
            continue;
        const double unit = qpair_variant( bucket, R, pinned_mb, pinned_c, pinned_h, pinned_g8 ).cost;
        if( unit <= 0 && !pinned )
            continue;                   // not measured
        const double c = (double) P * (unit > 0 ? unit : 1.0);
        if( c < best_cost ) {
            best_cost = c;
            best_r = R;
            *passes = P;
        }
    }
    if( best_r == 0 && pinned )         // the pinned R does not fit this query
        return choose_qpair_rows( Q, passes, 0, bucket, pinned_mb, pinned_c, pinned_h, pinned_g8 );
    if( best_r == 0 ) {                 // an empty table: 20 rows per thread
        best_r = 20;
        *passes = std::max<uint32_t>( 1, (Q + QP_G * 20 - 1) / (QP_G * 20) );
    }
    return best_r;
}

void Engine::run_qpair_entry( const SearchRequest & req, uint32_t nq, PairTask * next, unsigned * next_count,
        uint32_t cap, const std::vector<uint32_t> * slots, uint32_t seq_lo, uint32_t seq_hi ) {
    // the sequences order_desc[seq_lo, seq_hi) (all by default)
    const uint32_t n_all = (uint32_t) db_.order_desc.size();
    const uint32_t lo = std::min( seq_lo, n_all ), hi = std::min( seq_hi, n_all );
    const uint32_t n_seq = hi - lo;
    if( n_seq == 0 )
        return;
    const bool nw = req.algo == 1;
    // pair the queries that fit, longest first; longer ones run the emulation
    std::vector<uint32_t> fit, fallback;
    if( slots ) {
        for( uint32_t s : *slots )
            (h_qlen_[s] <= FAST_MAX_ROWS ? fit : fallback).push_back( s );
    }
    else {
        for( uint32_t s = 0; s < nq; s++ )
            (h_qlen_[s] <= FAST_MAX_ROWS ? fit : fallback).push_back( s );
    }
    std::stable_sort( fit.begin(), fit.end(), [&]( uint32_t a, uint32_t b ) { return h_qlen_[a] > h_qlen_[b]; } );
    const uint32_t n_qp = (uint32_t) ((fit.size() + 1) / 2);
    // SSA_B200_QP_R=16|20|24|28 and SSA_B200_QP_MB=4|5 pin the shape (tuning)
    const char * pin = getenv( "SSA_B200_QP_R" );
    const int pinned_r = pin ? atoi( pin ) : 0;
    const char * pin_mb = getenv( "SSA_B200_QP_MB" );
    const int pinned_mb = pin_mb ? atoi( pin_mb ) : 0;
    const char * pin_c = getenv( "SSA_B200_QP_C" );      // 2|4 columns per step
    const int pinned_c = pin_c ? atoi( pin_c ) : 0;
    const char * pin_h = getenv( "SSA_B200_QP_HMAX" );   // 0|1 running maximum in fp16x2
    const int pinned_h = pin_h ? (atoi( pin_h ) ? 1 : 0) : -1;
    const char * pin_g8 = getenv( "SSA_B200_QP_G8" );    // 0|1 8 threads per sequence (R = 24)
    const int pinned_g8 = pin_g8 ? (atoi( pin_g8 ) ? 1 : 0) : -1;
    // the database bucket of the shape table: these sequences' mean length and count
    uint64_t seq_res = 0;
    for( uint32_t i = lo; i < hi; i++ )
        seq_res += db_.len[db_.order_desc[i]];
    const int bucket = db_bucket( (double) seq_res / std::max<uint32_t>( 1, n_seq ), n_seq );
    std::vector<uint32_t> qp_slots( 2 * std::max<uint32_t>( 1, n_qp ), 0xffffffffu );
    std::vector<uint32_t> qp_rows( std::max<uint32_t>( 1, n_qp ), 0 );
    std::vector<uint64_t> qp_off( std::max<uint32_t>( 1, n_qp ), 0 );
    std::vector<std::vector<uint32_t>> by_r( 4 );     // R = 16, 20, 24, 28
    uint64_t total = 0;
    for( uint32_t i = 0; i < n_qp; i++ ) {
        qp_slots[2 * i] = fit[2 * i];
        if( 2 * i + 1 < fit.size() )
            qp_slots[2 * i + 1] = fit[2 * i + 1];
        uint32_t P = 1;
        const int R = choose_qpair_rows( h_qlen_[fit[2 * i]], &P, pinned_r, bucket, pinned_mb, pinned_c, pinned_h,
                pinned_g8 );
        qp_rows[i] = P * (uint32_t) (QP_G * R);
        by_r[R / 4 - 4].push_back( i );
    }
    // NW: per pair, the longest sequence whose matrix (padded rows and the last
    // block's pad columns included) stays within +-30000: every step of a path
    // changes a value by at most m, and a path has at most rows + L + 4 steps
    // and two gap openings
    std::vector<uint32_t> qp_lmax( std::max<uint32_t>( 1, n_qp ), 0 );
    if( nw ) {
        int64_t m = std::max<int64_t>( 1, std::llabs( (int64_t) req.gap_extend ) );
        for( int c = 0; c < 1024; c++ )
            m = std::max<int64_t>( m, std::llabs( (int64_t) (int16_t) req.matrix[c] ) );
        const int64_t budget = 30000 - 2 * std::llabs( (int64_t) req.gap_open );
        for( uint32_t i = 0; i < n_qp; i++ ) {
            const int64_t l = budget / m - (int64_t) qp_rows[i] - 4;
            qp_lmax[i] = (uint32_t) std::max<int64_t>( 0, l );
        }
    }
    // profiles: QP_CODES x rows words per pair (16-byte aligned: rows % 16 == 0)
    for( int ri = 0; ri < 4; ri++ )
        for( uint32_t i : by_r[ri] ) {
            qp_off[i] = total;
            total += (uint64_t) QP_CODES * qp_rows[i];
        }
    std::vector<uint32_t> units;                  // pairs grouped by class, longest first
    for( auto & v : by_r ) {
        std::stable_sort( v.begin(), v.end(), [&]( uint32_t a, uint32_t b ) { return qp_rows[a] > qp_rows[b]; } );
        units.insert( units.end(), v.begin(), v.end() );
    }
    d_qp_prof_.ensure( std::max<uint64_t>( total, 4 ) * sizeof(uint32_t) );
    d_qp_off_.ensure( qp_off.size() * sizeof(uint64_t) );
    d_qp_rows_.ensure( qp_rows.size() * sizeof(uint32_t) );
    d_qp_slots_.ensure( qp_slots.size() * sizeof(uint32_t) );
    d_qp_units_.ensure( std::max<size_t>( 1, units.size() ) * sizeof(uint32_t) );
    d_qp_lmax_.ensure( qp_lmax.size() * sizeof(uint32_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_qp_lmax_.p, qp_lmax.data(), qp_lmax.size() * sizeof(uint32_t),
            cudaMemcpyHostToDevice, stream_ ) );
    unsigned * redo_count = d_counts_.as<unsigned>() + 5;
    if( nw )
        CUDA_CHECK( cudaMemsetAsync( redo_count, 0, sizeof(unsigned), stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qp_off_.p, qp_off.data(), qp_off.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
            stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qp_rows_.p, qp_rows.data(), qp_rows.size() * sizeof(uint32_t),
            cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qp_slots_.p, qp_slots.data(), qp_slots.size() * sizeof(uint32_t),
            cudaMemcpyHostToDevice, stream_ ) );
    if( !units.empty() )
        CUDA_CHECK( cudaMemcpyAsync( d_qp_units_.p, units.data(), units.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice, stream_ ) );
    if( n_qp ) {
        CUDA_CHECK( launch_build_profile_qp( d_qcodes_.as<uint8_t>(), d_qoff_.as<uint64_t>(), d_qlen_.as<uint32_t>(),
                d_qp_slots_.as<uint32_t>(), n_qp, d_qp_rows_.as<uint32_t>(), d_matrix_.as<int64_t>(),
                d_qp_prof_.as<uint32_t>(), d_qp_off_.as<uint64_t>(), nw ? 16 : 8, stream_ ) );
        launches_++;
    }

    // work units: ranges of length-sorted sequences (multiples of QP_GPW)
    // holding about equal numbers of columns, the longest first; every pair of
    // a class gets every range.  A warp takes one unit at a time.
    uint64_t total_cols = 0;
    for( uint32_t i = lo; i < hi; i++ )
        total_cols += (db_.len[db_.order_desc[i]] + 3u) & ~3u;
    const uint64_t want_units = (uint64_t) sms_ * 16 * 24;
    const uint64_t target = std::max<uint64_t>( 1, total_cols * std::max<uint32_t>( 1, n_qp ) / want_units );
    std::vector<uint32_t> bounds{ 0 };
    {
        uint64_t acc = 0;
        for( uint32_t i = 0; i < n_seq; i++ ) {
            acc += (db_.len[db_.order_desc[lo + i]] + 3u) & ~3u;
            if( acc >= target && (i + 1) % QP_GPW == 0 ) {
                bounds.push_back( i + 1 );
                acc = 0;
            }
        }
        if( bounds.back() != n_seq )
            bounds.push_back( n_seq );
    }
    const uint32_t n_chunks = (uint32_t) bounds.size() - 1;
    d_bounds_.ensure( bounds.size() * sizeof(uint32_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_bounds_.p, bounds.data(), bounds.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
            stream_ ) );
    CUDA_CHECK( cudaEventRecord( ev_ready_, stream_ ) );
    const uint32_t scratch_cols = (((db_.max_len + 3u) & ~3u) >> 1) + 2u;
    const bool timing = getenv( "SSA_B200_TIMING" ) != nullptr;
    uint64_t seg_residues = 0;
    for( uint32_t i = lo; i < hi; i++ )
        seg_residues += db_.len[db_.order_desc[i]];
    // classes launched heaviest first (most rows per thread: the longest
    // queries), so that the last class to finish is the lightest
    size_t class_start[4] = { 0, 0, 0, 0 };
    for( int ri = 1; ri < 4; ri++ )
        class_start[ri] = class_start[ri - 1] + by_r[ri - 1].size();
    for( int k = 0; k < 4; k++ ) {
        const int ri = 3 - k;
        const size_t class_first = class_start[ri];
        const std::vector<uint32_t> & cls = by_r[ri];
        if( cls.empty() )
            continue;
        const int R = 4 * (ri + 4);
        // Needleman-Wunsch: 4 columns per step unless SSA_B200_QP_C=2 pins the
        // 2-column kernel (4 resident CTAs per SM either way)
        const QpVariant var = nw ? QpVariant{ 4, pinned_c == 2 ? 2 : 4, false, false, 0 }
                                 : qpair_variant( bucket, R, pinned_mb, pinned_c, pinned_h, pinned_g8 );
        const int mb = var.mb;
        auto launch = [&]( const QPairParams & pp, int grid, int * per ) {
            if( nw )
                return var.cols == 4 ? launch_nw_qpair4( R, pp, grid, class_stream_[ri], per )
                                     : launch_nw_qpair( R, pp, grid, class_stream_[ri], per );
            return var.cols == 4 ? launch_sw_qpair4( R, mb, var.hmax, var.g8, pp, grid, class_stream_[ri], per )
                                 : launch_sw_qpair( R, mb, pp, grid, class_stream_[ri], per );
        };
        bool multi = false;
        for( uint32_t i : cls )
            multi |= qp_rows[i] > (uint32_t) (QP_G * R);
        last_shapes_.push_back( { nw ? (var.cols == 4 ? "nw_qpair4" : "nw_qpair") : var.hmax ? "sw_qpair4h"
                : var.g8 ? "sw_qpair4g8"
                : var.cols == 4 ? "sw_qpair4" : "sw_qpair", R, mb,
                (uint32_t) cls.size(), bucket } );
        QPairParams p{};
        int per_sm = 0;
        CUDA_CHECK( launch( p, 0, &per_sm ) );
        const int grid = sms_ * std::max( 1, per_sm );
        CUDA_CHECK( cudaStreamWaitEvent( class_stream_[ri], ev_ready_, 0 ) );
        unsigned long long * unit_counter = d_counts_.as<unsigned long long>() + 8 + ri;   // bytes 64..95
        CUDA_CHECK( cudaMemsetAsync( unit_counter, 0, sizeof(unsigned long long), class_stream_[ri] ) );
        p.db = db_view();
        p.order = d_order_.as<uint32_t>() + lo;
        p.prof = d_qp_prof_.as<uint32_t>();
        p.prof_off = d_qp_off_.as<uint64_t>();
        p.qp_slots = d_qp_slots_.as<uint32_t>();
        p.qp_rows = d_qp_rows_.as<uint32_t>();
        p.unit_pairs = d_qp_units_.as<uint32_t>() + class_first;
        p.n_class = (uint32_t) cls.size();
        p.n_chunks = n_chunks;
        p.chunk_bounds = d_bounds_.as<uint32_t>();
        p.n_units = (uint64_t) n_chunks * cls.size();
        p.unit_counter = unit_counter;
        // the 8-bit Smith-Waterman lanes add the int8 truncation of gapO + gapE
        p.gap_oe = nw ? req.gap_open + req.gap_extend : (int8_t) (req.gap_open + req.gap_extend);
        p.gap_e = req.gap_extend;
        p.sink.score = score_sink();
        p.sink.score_stride = db_.n_ids;
        p.sink.next = next;
        p.sink.next_count = next_count;
        p.sink.next_cap = cap;
        p.sink.error_flags = d_counts_.as<unsigned>() + 2;
        if( multi ) {
            p.scratch = (int4 *) d_scratch_fast_[ri].ensure( (size_t) grid * (QP_THREADS_PER_CTA / 32) * QP_GPW *
                    scratch_cols * sizeof(int4) );
            p.scratch_cols = scratch_cols;
        }
        p.gap_open = req.gap_open;
        p.qlen = d_qlen_.as<uint32_t>();
        p.qp_lmax = d_qp_lmax_.as<uint32_t>();
        p.redo = d_list_b_.as<PairTask>();
        p.redo_count = redo_count;
        p.redo_cap = cap;
        if( timing )
            CUDA_CHECK( cudaEventRecord( ev_cls_t_[2 * ri], class_stream_[ri] ) );
        CUDA_CHECK( launch( p, grid, nullptr ) );
        launches_++;
        if( timing )
            CUDA_CHECK( cudaEventRecord( ev_cls_t_[2 * ri + 1], class_stream_[ri] ) );
        CUDA_CHECK( cudaEventRecord( ev_class_[ri], class_stream_[ri] ) );
        CUDA_CHECK( cudaStreamWaitEvent( stream_, ev_class_[ri], 0 ) );
    }
    if( timing ) {
        for( int ri = 0; ri < 4; ri++ ) {
            if( by_r[ri].empty() )
                continue;
            float ms = 0;
            CUDA_CHECK( cudaEventSynchronize( ev_cls_t_[2 * ri + 1] ) );
            CUDA_CHECK( cudaEventElapsedTime( &ms, ev_cls_t_[2 * ri], ev_cls_t_[2 * ri + 1] ) );
            double cells = 0, padded = 0;
            for( uint32_t i : by_r[ri] ) {
                const uint32_t a = qp_slots[2 * i], b = qp_slots[2 * i + 1];
                cells += (double) (h_qlen_[a] + (b == 0xffffffffu ? 0u : h_qlen_[b])) * (double) seg_residues;
                padded += 2.0 * qp_rows[i] * (double) total_cols;
            }
            fprintf( stderr, "[ssa timing] qpair class R=%d: %zu pairs, %.3f ms, %.3e cells (%.1f%% of computed), "
                    "%.1f GCUPS\n", 4 * (ri + 4), by_r[ri].size(), ms, cells, 100.0 * cells / padded,
                    cells / (ms * 1e-3) / 1e9 );
        }
    }
    if( nw ) {
        // sequences beyond a pair's exact range: the 16-bit lane emulation
        unsigned n_redo = 0;
        CUDA_CHECK( cudaMemcpyAsync( &n_redo, redo_count, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        n_redo = std::min( n_redo, cap );
        if( n_redo )
            run_pass( 1, 16, req, nq, d_list_b_.as<PairTask>(), n_redo, false, next, next_count, cap );
    }
    if( !fallback.empty() ) {
        d_slots_.ensure( fallback.size() * sizeof(uint32_t) );
        CUDA_CHECK( cudaMemcpyAsync( d_slots_.p, fallback.data(), fallback.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice, stream_ ) );
        run_pass( req.algo, req.bit_width, req, nq, nullptr, (uint64_t) fallback.size() * n_seq, true, next,
                next_count, cap, d_slots_.as<uint32_t>(), (uint32_t) fallback.size(), lo );
    }
}

void Engine::search( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & groups_in, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    init_device();
    const HostDb & db = database();
    serving_ = false;
    serve_layout_ = false;      // the query buffers are reused for this batch
    // groups of query sequences (strands or frames of one query)
    std::vector<uint32_t> groups = groups_in;
    if( groups.empty() )
        groups.assign( queries.size(), 1u );
    std::vector<uint64_t> gstart( groups.size() + 1, 0 );
    for( size_t g = 0; g < groups.size(); g++ )
        gstart[g + 1] = gstart[g] + groups[g];
    if( gstart.back() != queries.size() )
        fatal( "Internal error: query groups do not cover the queries." );
    out.assign( groups.size(), {} );
    stats.query_overflow.assign( groups.size(), { 0, 0 } );
    last_shapes_.clear();
    if( queries.empty() )
        return;
    const uint64_t n_ne = db.order_desc.size();

    // matrix on the device
    d_matrix_.ensure( 1024 * sizeof(int64_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_matrix_.p, req.matrix, 1024 * sizeof(int64_t), cudaMemcpyHostToDevice, stream_ ) );

    // the 64-bit pass in int64 arithmetic when the values can leave the int32 range
    {
        uint32_t qmax = 0;
        for( const QueryCodes & q : queries )
            qmax = std::max( qmax, q.len );
        wide_ = needs_int64( req, qmax, db.max_len );
    }
    // sub-batches bounded by the per-pair result memory (int32 scores, plus
    // int64 ones in the wide case)
    const uint64_t pair_budget = this->pair_budget();
    const uint64_t per_query = std::max<uint64_t>( 1, std::max<uint64_t>( n_ne, db.n_ids ) );
    const size_t batch = (size_t) std::max<uint64_t>(
            1, std::min<uint64_t>( std::min<uint64_t>( queries.size(), pair_budget / per_query ), 65535 ) );

    CUDA_CHECK( cudaEventRecord( ev0_, stream_ ) );
    for( size_t g0 = 0; g0 < groups.size(); ) {
        // whole groups, at most `batch` query sequences (at least one group)
        size_t g1 = g0 + 1;
        while( g1 < groups.size() && gstart[g1 + 1] - gstart[g0] <= batch )
            g1++;
        const size_t b0 = gstart[g0];
        const uint32_t nq = (uint32_t) (gstart[g1] - b0);
        // ---- upload queries
        upload_queries( queries.data() + b0, nq, true, stats );
        for( uint32_t q = 0; q < nq; q++ )
            stats.cells += (uint64_t) h_qlen_[q] * db.residues;

        // ---- result and re-queue buffers
        const uint64_t n_pairs = (uint64_t) nq * n_ne;
        const size_t score_bytes = (size_t) nq * db.n_ids * sizeof(int32_t);
        d_score_.ensure( std::max<size_t>( score_bytes, 4 ) );
        if( wide_ )
            d_score64_.ensure( std::max<size_t>( 2 * score_bytes, 8 ) );
        // re-queue lists sized for the overflows a search expects (a few per
        // query): 1/32 of the pairs, at least 4M entries; an entry pass that
        // re-queues more runs again with lists of its count
        const uint64_t all_pairs = std::min<uint64_t>( std::max<uint64_t>( n_pairs, 1 ), 0xffffffffull );
        uint32_t cap = (uint32_t) std::min<uint64_t>( all_pairs, std::max<uint64_t>( (uint64_t) 1 << 22,
                all_pairs >> 5 ) );
        if( const char * c0 = getenv( "SSA_B200_REQUEUE_CAP" ) )   // a smaller first size (tests of the regrowth)
            cap = (uint32_t) std::max<uint64_t>( 1, std::min<uint64_t>( cap, strtoull( c0, nullptr, 10 ) ) );
        d_list_a_.ensure( (size_t) cap * sizeof(PairTask) );
        d_list_b_.ensure( (size_t) cap * sizeof(PairTask) );
        d_counts_.ensure( 32 * sizeof(unsigned long long) );
        CUDA_CHECK( cudaMemsetAsync( d_counts_.p, 0, 32 * sizeof(unsigned long long), stream_ ) );
        unsigned * cnt = d_counts_.as<unsigned>();   // [0] list a, [1] list b, [2] errors, [5] NW redo

        // ---- passes
        const bool timing = getenv( "SSA_B200_TIMING" ) != nullptr;
        CUDA_CHECK( cudaEventRecord( ev_phase_[0], stream_ ) );
        const int entry = req.bit_width;
        std::vector<PairTask> list_entry, list_16;   // host copies for the replay
        uint64_t n_a = 0, n_b = 0;
        float entry_ms = 0;     // the entry passes of all segments
        // a resident database is one segment; a streamed one runs the entry pass
        // and the cascade of each segment while it is on the device
        const uint32_t n_seg = streaming_ ? (uint32_t) seg_lo_.size() : 1;
        for( uint32_t sg = 0; sg < n_seg; sg++ ) {
            const uint32_t lo = streaming_ ? seg_lo_[sg] : 0;
            const uint32_t hi = streaming_ ? seg_hi_[sg] : (uint32_t) n_ne;
            if( streaming_ ) {
                make_resident( sg, stats );
                CUDA_CHECK( cudaMemsetAsync( cnt, 0, 2 * sizeof(unsigned), stream_ ) );
            }
            const uint64_t seg_pairs = (uint64_t) nq * (hi - lo);
            CUDA_CHECK( cudaEventRecord( ev_seg_[0], stream_ ) );
            auto run_entry = [&]() {
                if( (fast_eligible( req ) && (nq >= 2 || streaming_) && !getenv( "SSA_B200_NO_QPAIR" )) ||
                        nw_fast_eligible( req ) )
                    run_qpair_entry( req, nq, d_list_a_.as<PairTask>(), cnt + 0, cap, nullptr, lo, hi );
                else if( fast_eligible( req ) )
                    run_fast_entry( req, nq, d_list_a_.as<PairTask>(), cnt + 0, cap );
                else
                    run_pass( req.algo, entry, req, nq, nullptr, seg_pairs, true, d_list_a_.as<PairTask>(), cnt + 0,
                            cap, nullptr, 0, lo );
            };
            run_entry();
            for( ;; ) {
                // counts of the entry list and the NW redo list (their atomic
                // counters count every append, kept or not) and the error flags
                unsigned c[6] = {};
                CUDA_CHECK( cudaMemcpyAsync( c, cnt, sizeof c, cudaMemcpyDeviceToHost, stream_ ) );
                CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
                const uint64_t need = std::max<uint64_t>( c[0], c[5] );
                if( need <= cap && !(c[2] & ERR_REQUEUE_OVERFLOW) )
                    break;
                cap = (uint32_t) std::min<uint64_t>( all_pairs, std::max<uint64_t>( need, 2ull * cap ) );
                d_list_a_.ensure( (size_t) cap * sizeof(PairTask) );
                d_list_b_.ensure( (size_t) cap * sizeof(PairTask) );
                CUDA_CHECK( cudaMemsetAsync( cnt, 0, 6 * sizeof(unsigned), stream_ ) );
                run_entry();
            }
            CUDA_CHECK( cudaEventRecord( ev_seg_[1], stream_ ) );
            CUDA_CHECK( cudaEventSynchronize( ev_seg_[1] ) );
            float seg_ms = 0;
            CUDA_CHECK( cudaEventElapsedTime( &seg_ms, ev_seg_[0], ev_seg_[1] ) );
            entry_ms += seg_ms;
            if( entry == 64 )
                continue;
            unsigned sa = 0, sb = 0;
            CUDA_CHECK( cudaMemcpyAsync( &sa, cnt + 0, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
            CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
            sa = std::min( sa, cap );
            if( sa == 0 )
                continue;
            const int w2 = (entry == 8) ? 16 : 64;
            PairTask * nx = (w2 == 16) ? d_list_b_.as<PairTask>() : nullptr;
            run_pass( req.algo, w2, req, nq, d_list_a_.as<PairTask>(), sa, false, nx, cnt + 1, cap );
            if( w2 == 16 ) {
                CUDA_CHECK( cudaMemcpyAsync( &sb, cnt + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
                CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
                sb = std::min( sb, cap );
                if( sb )
                    run_pass( req.algo, 64, req, nq, d_list_b_.as<PairTask>(), sb, false, nullptr, cnt + 3, 0 );
            }
            list_entry.resize( n_a + sa );
            CUDA_CHECK( cudaMemcpyAsync( list_entry.data() + n_a, d_list_a_.p, sa * sizeof(PairTask),
                    cudaMemcpyDeviceToHost, stream_ ) );
            if( sb ) {
                list_16.resize( n_b + sb );
                CUDA_CHECK( cudaMemcpyAsync( list_16.data() + n_b, d_list_b_.p, sb * sizeof(PairTask),
                        cudaMemcpyDeviceToHost, stream_ ) );
            }
            n_a += sa;
            n_b += sb;
            if( streaming_ )
                CUDA_CHECK( cudaStreamSynchronize( stream_ ) );   // the lists are reused by the next segment
        }
        CUDA_CHECK( cudaEventRecord( ev_phase_[2], stream_ ) );
        stats.d2h_bytes += score_bytes + (n_a + n_b) * sizeof(PairTask);
        int32_t * hs = (int32_t *) h_score_.ensure( std::max<size_t>( score_bytes, 4 ) );
        if( score_bytes )
            CUDA_CHECK( cudaMemcpyAsync( hs, d_score_.p, score_bytes, cudaMemcpyDeviceToHost, stream_ ) );
        int64_t * hs64 = nullptr;
        if( wide_ && score_bytes ) {
            hs64 = (int64_t *) h_score64_.ensure( 2 * score_bytes );
            CUDA_CHECK( cudaMemcpyAsync( hs64, d_score64_.p, 2 * score_bytes, cudaMemcpyDeviceToHost, stream_ ) );
            stats.d2h_bytes += 2 * score_bytes;
        }
        unsigned err = 0;
        CUDA_CHECK( cudaMemcpyAsync( &err, cnt + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaEventRecord( ev_phase_[3], stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        if( err )
            fatal( "Internal error in the GPU search (flags 0x%x).", err );
        const auto t_replay0 = std::chrono::steady_clock::now();

        // ---- host replay, one query (group of query sequences) per worker
        std::vector<ReplayQuery> rq( nq );
        for( uint32_t s = 0; s < nq; s++ ) {
            rq[s].score = hs + (size_t) s * db.n_ids;
            if( hs64 )
                rq[s].score64 = hs64 + (size_t) s * db.n_ids;
        }
        for( const PairTask & t : list_entry )
            rq[t.qslot].ovf_entry.emplace_back( t.id, t.nb_prev );
        for( const PairTask & t : list_16 )
            rq[t.qslot].ovf16.emplace_back( t.id, t.nb_prev );
        for( auto & r : rq ) {
            std::sort( r.ovf_entry.begin(), r.ovf_entry.end() );
            std::sort( r.ovf16.begin(), r.ovf16.end() );
        }
        const uint32_t * rank_entry = (entry == 64) ? nullptr : ranks( req.chunk_size, entry == 8 ? req.lanes8 : req.lanes16 );
        {
            const uint32_t ng = (uint32_t) (g1 - g0);
            const unsigned hw = std::max( 1u, std::thread::hardware_concurrency() );
            const unsigned nthreads = std::min<unsigned>( hw, ng );
            std::atomic<uint32_t> next{ 0 };
            std::vector<ReplayCounts> counts( ng );
            auto work = [&]() {
                for( ;; ) {
                    const uint32_t i = next.fetch_add( 1 );
                    if( i >= ng )
                        break;
                    const size_t g = g0 + i;
                    const uint32_t s0 = (uint32_t) (gstart[g] - b0);
                    if( groups[g] == 1 && db.upi == 1 )
                        replay_query( db, req, rq[s0], rank_entry, out[g], counts[i] );
                    else
                        replay_frames( db, req, &rq[s0], groups[g], out[g], counts[i] );
                }
            };
            if( nthreads <= 1 ) {
                work();
            }
            else {
                std::vector<std::thread> th;
                for( unsigned k = 0; k < nthreads; k++ )
                    th.emplace_back( work );
                for( auto & t : th )
                    t.join();
            }
            for( uint32_t i = 0; i < ng; i++ ) {
                stats.overflow8 += counts[i].overflow8;
                stats.overflow16 += counts[i].overflow16;
                stats.query_overflow[g0 + i] = { counts[i].overflow8, counts[i].overflow16 };
            }
        }
        const auto t_replay1 = std::chrono::steady_clock::now();
        CUDA_CHECK( cudaEventRecord( ev_phase_[4], stream_ ) );
        if( req.align_type == COMPUTE_ALIGNMENT ) {
            std::vector<std::pair<uint32_t, uint32_t>> lists;   // (out index, slot of its first sequence)
            for( size_t g = g0; g < g1; g++ )
                lists.emplace_back( (uint32_t) g, (uint32_t) (gstart[g] - b0) );
            traceback( req, out, lists, stats );
        }
        CUDA_CHECK( cudaEventRecord( ev_phase_[5], stream_ ) );
        {
            CUDA_CHECK( cudaEventSynchronize( ev_phase_[5] ) );
            float ms[5];
            // [0] entry passes, [1] cascades (and segment copies), [2] result copies, [3] traceback
            float passes = 0;
            CUDA_CHECK( cudaEventElapsedTime( &passes, ev_phase_[0], ev_phase_[2] ) );
            ms[0] = entry_ms;
            ms[1] = std::max( 0.0f, passes - entry_ms );
            CUDA_CHECK( cudaEventElapsedTime( &ms[2], ev_phase_[2], ev_phase_[3] ) );
            CUDA_CHECK( cudaEventElapsedTime( &ms[3], ev_phase_[4], ev_phase_[5] ) );
            const double rep = std::chrono::duration<double, std::milli>( t_replay1 - t_replay0 ).count();
            stats.entry_seconds += ms[0] * 1e-3;
            stats.kernel_seconds += (ms[0] + ms[1] + ms[3]) * 1e-3;
            if( timing )
            fprintf( stderr,
                    "[ssa timing] queries %u pairs %llu: entry %.3f ms, cascade %.3f ms (%llu+%llu re-queued), "
                    "copies %.3f ms, replay %.3f ms, traceback %.3f ms\n",
                    nq, (unsigned long long) n_pairs, ms[0], ms[1], (unsigned long long) n_a,
                    (unsigned long long) n_b, ms[2], rep, ms[3] );
        }
        g0 = g1;
    }
    CUDA_CHECK( cudaEventRecord( ev1_, stream_ ) );
    CUDA_CHECK( cudaEventSynchronize( ev1_ ) );
    float ms = 0;
    CUDA_CHECK( cudaEventElapsedTime( &ms, ev0_, ev1_ ) );
    stats.seconds_gpu += ms * 1e-3;
    stats.kernel_launches = launches_.load();
}

// Query codes of one batch to the device (slot s = queries[s]); profiles: also
// size the int32 profile buffer of the lane emulation.
void Engine::upload_queries( const QueryCodes * queries, uint32_t nq, bool profiles, SearchStats & stats ) {
    h_qoff_.assign( nq, 0 );
    h_qlen_.assign( nq, 0 );
    h_qpad_.assign( nq, 0 );
    h_prof_off_.assign( nq, 0 );
    uint64_t qtotal = 0, ptotal = 0;
    max_qlen_ = 0;
    for( uint32_t s = 0; s < nq; s++ ) {
        const QueryCodes & q = queries[s];
        h_qoff_[s] = qtotal;
        h_qlen_[s] = q.len;
        h_qpad_[s] = std::max<uint32_t>( 256, (q.len + 255u) & ~255u );
        h_prof_off_[s] = ptotal;
        qtotal += (q.len + 15u) & ~15u;
        ptotal += 32ull * h_qpad_[s];
        max_qlen_ = std::max( max_qlen_, q.len );
    }
    std::vector<uint8_t> hq( qtotal + 16, 0 );
    for( uint32_t s = 0; s < nq; s++ )
        memcpy( hq.data() + h_qoff_[s], queries[s].codes, queries[s].len );
    d_qcodes_.ensure( hq.size() );
    d_qoff_.ensure( nq * sizeof(uint64_t) );
    d_qlen_.ensure( nq * sizeof(uint32_t) );
    d_qpad_.ensure( nq * sizeof(uint32_t) );
    d_prof_off_.ensure( nq * sizeof(uint64_t) );
    if( profiles )
        d_prof_.ensure( ptotal * sizeof(int32_t) );
    stats.h2d_bytes += hq.size() + nq * (2 * sizeof(uint64_t) + 2 * sizeof(uint32_t));
    CUDA_CHECK( cudaMemcpyAsync( d_qcodes_.p, hq.data(), hq.size(), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qoff_.p, h_qoff_.data(), nq * sizeof(uint64_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qlen_.p, h_qlen_.data(), nq * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qpad_.p, h_qpad_.data(), nq * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_prof_off_.p, h_prof_off_.data(), nq * sizeof(uint64_t), cudaMemcpyHostToDevice,
            stream_ ) );
    prof_width_ = -1;
}

// Warps per hit in the traceback passes (stripe_pipeline.cuh): 4 for at least
// 4 stripes of query rows and 8M cells, 2 for at least 2 stripes (they run
// side by side instead of one after the other), else 1.
static int tb_group( uint32_t rows, uint32_t cols ) {
    const uint32_t stripes = (rows + 32u * TB_WORD_ROWS - 1) / (32u * TB_WORD_ROWS);
    if( stripes >= 4 && (uint64_t) rows * cols >= ((uint64_t) 1 << 23) )
        return 4;
    return stripes >= 2 ? 2 : 1;
}

// Largest magnitude of one DP step: a score-table entry or a gap cost.
static int64_t max_abs_step( const SearchRequest & req ) {
    int64_t m = std::llabs( (int64_t) req.gap_open ) + std::llabs( (int64_t) req.gap_extend );
    for( int k = 0; k < 1024; k++ )
        m = std::max<int64_t>( m, std::llabs( req.matrix[k] ) );
    return m;
}

void Engine::traceback( const SearchRequest & req, std::vector<std::vector<Hit>> & out,
        const std::vector<std::pair<uint32_t, uint32_t>> & lists, SearchStats & stats, bool scores_from_regions ) {
    std::vector<TbHit> hits;
    std::vector<std::pair<uint32_t, uint32_t>> where;   // (list index, hit index)
    for( const auto & l : lists ) {
        auto & hl = out[l.first];
        for( uint32_t k = 0; k < hl.size(); k++ ) {
            // the hit's query sequence; the database record's first unit (the
            // reference aligns a reverse-complement hit on the forward strand:
            // src/util/util_sequence.c:384-402)
            const uint32_t fwd_unit = hl[k].unit - hl[k].unit % db_.upi;
            hits.push_back( TbHit{ l.second + hl[k].q_index, fwd_unit, (int32_t) hl[k].score, req.algo } );
            where.emplace_back( l.first, k );
        }
    }
    const uint32_t nh = (uint32_t) hits.size();
    if( nh == 0 )
        return;
    // the hits by warps per hit (4, 2, 1), each class largest first: the
    // kernels hand hits out in this order
    {
        std::vector<uint32_t> perm( nh );
        for( uint32_t h = 0; h < nh; h++ )
            perm[h] = h;
        auto work = [&]( uint32_t h ) { return (uint64_t) h_qlen_[hits[h].qslot] * db_.len[hits[h].id]; };
        auto group = [&]( uint32_t h ) { return tb_group( h_qlen_[hits[h].qslot], db_.len[hits[h].id] ); };
        std::stable_sort( perm.begin(), perm.end(), [&]( uint32_t a, uint32_t b ) {
            return group( a ) != group( b ) ? group( a ) > group( b ) : work( a ) > work( b );
        } );
        std::vector<TbHit> hs( nh );
        std::vector<std::pair<uint32_t, uint32_t>> ws( nh );
        for( uint32_t h = 0; h < nh; h++ ) {
            hs[h] = hits[perm[h]];
            ws[h] = where[perm[h]];
        }
        hits.swap( hs );
        where.swap( ws );
    }
    // value range guard: every DP value is bounded by (q + d) * max |step|
    const int64_t mabs = max_abs_step( req );
    std::vector<TbRegion> regions( nh );
    std::vector<uint64_t> last_off( nh + 1, 0 );
    for( uint32_t h = 0; h < nh; h++ ) {
        const uint32_t A = h_qlen_[hits[h].qslot], B = db_.len[hits[h].id];
        if( (int64_t) (A + B + 4) * (mabs + 1) * 2 > INT32_MAX )
            fatal( "Alignment of %u x %u residues exceeds the supported score range.", A, B );
        TbRegion rg{};
        if( req.algo == 1 ) {
            rg.a_begin = 0;
            rg.a_end = (int32_t) A - 1;
            rg.b_begin = 0;
            rg.b_end = (int32_t) B - 1;
            rg.status = (A && B) ? 0 : 1;
        }
        regions[h] = rg;
        last_off[h + 1] = last_off[h] + A;
    }
    TbParams p{};
    // the hits as the device sees them: with a streamed database their
    // sequences are gathered into a view of their own and renumbered
    std::vector<TbHit> dev_hits = hits;
    if( streaming_ ) {
        std::vector<uint32_t> ids;
        std::unordered_map<uint32_t, uint32_t> index;
        for( TbHit & t : dev_hits ) {
            auto it = index.find( t.id );
            if( it == index.end() ) {
                it = index.emplace( t.id, (uint32_t) ids.size() ).first;
                ids.push_back( t.id );
            }
            t.id = it->second;
        }
        p.db = gather_view( ids, stats );
    }
    else {
        p.db = db_view();
    }
    p.qcodes = d_qcodes_.as<uint8_t>();
    p.qoff = d_qoff_.as<uint64_t>();
    p.qlen = d_qlen_.as<uint32_t>();
    p.matrix = d_matrix_.as<int64_t>();
    p.gap_open = req.gap_open;
    p.gap_extend = req.gap_extend;
    p.error_flags = d_counts_.as<unsigned>() + 2;
    const int grid = sms_ * 2;
    const uint32_t cols = db_.max_len + 4;
    constexpr uint32_t stripe_rows = 32 * TB_WORD_ROWS;
    // boundary rows in global memory: one per group of warps (8, 4 and 2
    // groups per CTA of 256 threads for groups of 1, 2 and 4)
    int4 * scratch1 = max_qlen_ > stripe_rows ? (int4 *) d_scratch_.ensure( (size_t) grid * 8 * cols * sizeof(int4) )
                                              : nullptr;
    int4 * scratch2 = max_qlen_ > 2 * stripe_rows
            ? (int4 *) d_scratch2_.ensure( (size_t) grid * 4 * cols * sizeof(int4) ) : nullptr;
    int4 * scratch4 = max_qlen_ > 4 * stripe_rows
            ? (int4 *) d_scratch4_.ensure( (size_t) grid * 2 * cols * sizeof(int4) ) : nullptr;
    unsigned long long * counters = d_counts_.as<unsigned long long>() + 16;   // bytes 128..223
    // Launches one phase over the hits [0, n) of the current arrays: [0, k4) on
    // groups of 4 warps, [k4, k2) on groups of 2, [k2, n) on single warps, the
    // three classes concurrently on three streams.
    enum { TB_REGIONS, TB_PATHS, TB_FUSED };
    auto launch_split = [&]( int phase, uint32_t n, uint32_t k4, uint32_t k2, cudaEvent_t * ev ) {
        const uint32_t lo[3] = { 0, k4, k2 }, hi[3] = { k4, k2, n };
        const int group[3] = { 4, 2, 1 };
        int4 * scratch[3] = { scratch4, scratch2, scratch1 };
        cudaStream_t st[3] = { stream_, class_stream_[0], class_stream_[1] };
        CUDA_CHECK( cudaMemsetAsync( counters, 0, 12 * sizeof(unsigned long long), stream_ ) );
        CUDA_CHECK( cudaEventRecord( ev_ready_, stream_ ) );
        bool timed = false;
        for( int c = 0; c < 3; c++ ) {
            if( hi[c] <= lo[c] )
                continue;
            TbParams q = p;
            q.n_hits = hi[c] - lo[c];
            q.scratch = scratch[c];
            q.scratch_cols = scratch[c] ? cols : 0;
            q.hit_counters = counters + 4 * c;
            q.hits = p.hits + lo[c];
            q.regions = p.regions + lo[c];
            if( p.last_off )
                q.last_off = p.last_off + lo[c];
            if( p.dir_off ) {
                q.dir_off = p.dir_off + lo[c];
                q.ops_off = p.ops_off + lo[c];
                q.ops_len = p.ops_len + lo[c];
            }
            if( c > 0 )
                CUDA_CHECK( cudaStreamWaitEvent( st[c], ev_ready_, 0 ) );
            // events around the first class that runs (the largest hits)
            cudaEvent_t * e = timed ? nullptr : ev;
            timed = timed || ev != nullptr;
            CUDA_CHECK( phase == TB_REGIONS ? launch_tb_regions( q, group[c], grid, st[c], e )
                        : phase == TB_PATHS ? launch_tb_paths( q, group[c], grid, st[c], e )
                                            : launch_tb_fused( q, group[c], grid, st[c], e ) );
            if( c > 0 ) {
                CUDA_CHECK( cudaEventRecord( ev_class_[c], st[c] ) );
                CUDA_CHECK( cudaStreamWaitEvent( stream_, ev_class_[c], 0 ) );
            }
            launches_ += (phase == TB_FUSED) ? 3 : 2;
        }
    };
    // class bounds of hits sorted by warps per hit
    auto class_bounds = [&]( uint32_t n, auto group_of, uint32_t & k4, uint32_t & k2 ) {
        k4 = 0;
        while( k4 < n && group_of( k4 ) == 4 )
            k4++;
        k2 = k4;
        while( k2 < n && group_of( k2 ) == 2 )
            k2++;
    };
    const bool timing = getenv( "SSA_B200_TIMING" ) != nullptr;
    float t_fwd = 0, t_rev = 0, t_dir = 0, t_walk = 0;
    auto check_errors = [&]() {
        unsigned err = 0;
        CUDA_CHECK( cudaMemcpyAsync( &err, d_counts_.as<unsigned>() + 2, sizeof(unsigned), cudaMemcpyDeviceToHost,
                stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        if( err )
            fatal( "Internal error in the GPU traceback (flags 0x%x).", err );
    };

    // Smith-Waterman with a symmetric score table: the forward region pass and
    // the direction pass run as one sweep per hit (tb_fwddir_kernel), then the
    // reverse pass and the walk, wave by wave.  It needs every hit's last
    // database column past the initial E terms: (B - 1) x gapE < gapO + gapE
    // with B >= 2, and initial E and F values that are not above zero (gapO <= 0).
    bool fused = req.algo == 0 && req.gap_extend < 0 && req.gap_open <= 0;
    for( int d = 0; d < 32 && fused; d++ )
        for( int q = 0; q < 32 && fused; q++ )
            fused = req.matrix[(d << 5) + q] == req.matrix[(q << 5) + d];
    for( uint32_t h = 0; h < nh && fused; h++ )
        fused = db_.len[hits[h].id] >= 2 &&
                ((int64_t) db_.len[hits[h].id] - 1) * req.gap_extend < (int64_t) req.gap_open + req.gap_extend;
    int32_t * last_all = nullptr;
    if( fused ) {
        last_all = (int32_t *) d_tb_last_.ensure( 2 * last_off[nh] * sizeof(int32_t) + 16 );
        p.last_h = last_all;
        p.last_e = last_all + last_off[nh];
    }

    // ---- region phase (Smith-Waterman): end cell and begin cell of every hit
    if( req.algo == 0 && !fused ) {
        p.hits = (const TbHit *) d_tb_hits_.ensure( nh * sizeof(TbHit) );
        p.n_hits = nh;
        p.regions = (TbRegion *) d_tb_regions_.ensure( nh * sizeof(TbRegion) );
        int32_t * last = (int32_t *) d_tb_last_.ensure( 2 * last_off[nh] * sizeof(int32_t) + 16 );
        p.last_h = last;
        p.last_e = last + last_off[nh];
        p.last_off = (const uint64_t *) d_tb_last_off_.ensure( (nh + 1) * sizeof(uint64_t) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.hits, dev_hits.data(), nh * sizeof(TbHit), cudaMemcpyHostToDevice,
                stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( p.regions, regions.data(), nh * sizeof(TbRegion), cudaMemcpyHostToDevice,
                stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.last_off, last_off.data(), (nh + 1) * sizeof(uint64_t),
                cudaMemcpyHostToDevice, stream_ ) );
        uint32_t k4, k2;
        class_bounds( nh, [&]( uint32_t h ) { return tb_group( h_qlen_[hits[h].qslot], db_.len[hits[h].id] ); }, k4,
                k2 );
        launch_split( TB_REGIONS, nh, k4, k2, timing ? ev_tb_ : nullptr );
        CUDA_CHECK( cudaMemcpyAsync( regions.data(), p.regions, nh * sizeof(TbRegion), cudaMemcpyDeviceToHost,
                stream_ ) );
        check_errors();
        if( timing ) {
            CUDA_CHECK( cudaEventElapsedTime( &t_fwd, ev_tb_[0], ev_tb_[1] ) );
            CUDA_CHECK( cudaEventElapsedTime( &t_rev, ev_tb_[1], ev_tb_[2] ) );
        }
        stats.h2d_bytes += nh * (sizeof(TbHit) + sizeof(TbRegion) + sizeof(uint64_t));
        stats.d2h_bytes += nh * sizeof(TbRegion);
    }

    // ---- path phase: direction words (2 bits per cell of rows 0..a_end and
    // columns b_begin..b_end) and the walk, in waves whose direction words fit
    // the traceback memory
    std::vector<uint64_t> dir_words( nh, 0 ), ops_bytes( nh, 0 );
    uint64_t total_dir = 0;
    for( uint32_t h = 0; h < nh; h++ ) {
        TbRegion & rg = regions[h];
        if( fused ) {
            // the whole matrix: every query row and database column
            const uint32_t A = h_qlen_[hits[h].qslot], B = db_.len[hits[h].id];
            rg.dir_words = (int32_t) ((A + TB_WORD_ROWS - 1) / TB_WORD_ROWS);
            rg.dir_col0 = 0;
            dir_words[h] = (uint64_t) B * (uint64_t) rg.dir_words;
            ops_bytes[h] = (uint64_t) A + B + 1;
            total_dir += dir_words[h] * sizeof(uint16_t);
            continue;
        }
        if( rg.status == 2 )
            fatal( "Internal error in align function." );   // reference: src/algo/align.c:131
        if( rg.status != 0 )
            continue;
        // rows 0..a_end and columns b_begin..b_end
        rg.dir_words = (rg.a_end + TB_WORD_ROWS) / TB_WORD_ROWS;
        rg.dir_col0 = rg.b_begin;
        dir_words[h] = (uint64_t) (rg.b_end - rg.b_begin + 1) * (uint64_t) rg.dir_words;
        ops_bytes[h] = (uint64_t) (rg.a_end - rg.a_begin + 1) + (uint64_t) (rg.b_end - rg.b_begin + 1) + 1;
        total_dir += dir_words[h] * sizeof(uint16_t);
    }
    const uint64_t budget = traceback_budget();
    auto region_group = [&]( uint32_t h ) {
        if( fused )
            return tb_group( h_qlen_[hits[h].qslot], db_.len[hits[h].id] );
        const TbRegion & rg = regions[h];
        return rg.status == 0 ? tb_group( (uint32_t) rg.a_end + 1, (uint32_t) rg.b_end + 1 ) : 1;
    };
    // waves: consecutive runs of the hits in (more warps per hit first,
    // largest direction matrix first) order, each run as long as its matrices
    // fit
    std::vector<std::vector<uint32_t>> waves;
    {
        std::vector<uint32_t> order( nh );
        for( uint32_t h = 0; h < nh; h++ )
            order[h] = h;
        std::stable_sort( order.begin(), order.end(), [&]( uint32_t x, uint32_t y ) {
            const int gx = region_group( x ), gy = region_group( y );
            return gx != gy ? gx > gy : dir_words[x] > dir_words[y];
        } );
        uint64_t load = 0;
        for( uint32_t h : order ) {
            const uint64_t need = dir_words[h] * sizeof(uint16_t);
            if( waves.empty() || (load + need > budget && !waves.back().empty()) ) {
                waves.emplace_back();
                load = 0;
            }
            waves.back().push_back( h );
            load += need;
        }
    }
    for( const std::vector<uint32_t> & wave : waves ) {
        const uint32_t nw = (uint32_t) wave.size();
        std::vector<TbHit> whits( nw );
        std::vector<TbRegion> wregs( nw );
        std::vector<uint64_t> wdir( nw + 1, 0 ), wops( nw + 1, 0 ), wlast( nw, 0 );
        for( uint32_t k = 0; k < nw; k++ ) {
            whits[k] = dev_hits[wave[k]];
            wregs[k] = regions[wave[k]];
            wdir[k + 1] = wdir[k] + dir_words[wave[k]];
            wops[k + 1] = wops[k] + ops_bytes[wave[k]];
            wlast[k] = last_off[wave[k]];
        }
        if( fused ) {
            // the fused pass writes each hit's last column into its slice of
            // the last-row arrays of all hits
            p.last_off = (const uint64_t *) d_tb_last_off_.ensure( std::max<uint32_t>( 1, nw ) * sizeof(uint64_t) );
            CUDA_CHECK( cudaMemcpyAsync( (void *) p.last_off, wlast.data(), nw * sizeof(uint64_t),
                    cudaMemcpyHostToDevice, stream_ ) );
            stats.h2d_bytes += nw * sizeof(uint64_t);
        }
        p.hits = (const TbHit *) d_tb_hits_.ensure( nw * sizeof(TbHit) );
        p.n_hits = nw;
        p.regions = (TbRegion *) d_tb_regions_.ensure( nw * sizeof(TbRegion) );
        p.dirs = (uint16_t *) d_tb_dirs_.ensure( wdir[nw] * sizeof(uint16_t) + 16 );
        p.dir_off = (const uint64_t *) d_tb_dir_off_.ensure( (nw + 1) * sizeof(uint64_t) );
        p.ops = (char *) d_tb_ops_.ensure( wops[nw] + 16 );
        p.ops_off = (const uint64_t *) d_tb_ops_off_.ensure( (nw + 1) * sizeof(uint64_t) );
        p.ops_len = (uint32_t *) d_tb_ops_len_.ensure( nw * sizeof(uint32_t) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.hits, whits.data(), nw * sizeof(TbHit), cudaMemcpyHostToDevice,
                stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( p.regions, wregs.data(), nw * sizeof(TbRegion), cudaMemcpyHostToDevice, stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.dir_off, wdir.data(), (nw + 1) * sizeof(uint64_t),
                cudaMemcpyHostToDevice, stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.ops_off, wops.data(), (nw + 1) * sizeof(uint64_t),
                cudaMemcpyHostToDevice, stream_ ) );
        uint32_t k4, k2;
        class_bounds( nw, [&]( uint32_t k ) { return region_group( wave[k] ); }, k4, k2 );
        launch_split( fused ? TB_FUSED : TB_PATHS, nw, k4, k2, timing ? ev_tb_ + 2 : nullptr );
        std::vector<uint32_t> ops_len( nw );
        std::vector<char> ops( wops[nw] + 1 );
        CUDA_CHECK( cudaMemcpyAsync( ops_len.data(), p.ops_len, nw * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( ops.data(), p.ops, wops[nw], cudaMemcpyDeviceToHost, stream_ ) );
        if( fused || (scores_from_regions && req.algo == 1) ) {
            CUDA_CHECK( cudaMemcpyAsync( wregs.data(), p.regions, nw * sizeof(TbRegion), cudaMemcpyDeviceToHost,
                    stream_ ) );
            stats.d2h_bytes += nw * sizeof(TbRegion);
        }
        check_errors();
        if( fused ) {
            // the regions the fused and reverse passes found
            for( uint32_t k = 0; k < nw; k++ ) {
                if( wregs[k].status == 2 )
                    fatal( "Internal error in align function." );   // reference: src/algo/align.c:131
                regions[wave[k]] = wregs[k];
            }
        }
        else if( scores_from_regions && req.algo == 1 ) {
            for( uint32_t k = 0; k < nw; k++ )
                regions[wave[k]].fwd_score = wregs[k].fwd_score;
        }
        if( timing ) {
            float a = 0, b = 0;
            CUDA_CHECK( cudaEventElapsedTime( &a, ev_tb_[2], ev_tb_[3] ) );
            CUDA_CHECK( cudaEventElapsedTime( &b, ev_tb_[3], ev_tb_[4] ) );
            t_dir += a;
            t_walk += b;
        }
        stats.h2d_bytes += nw * (sizeof(TbHit) + sizeof(TbRegion) + 2 * sizeof(uint64_t));
        stats.d2h_bytes += nw * sizeof(uint32_t) + wops[nw];
        for( uint32_t k = 0; k < nw; k++ ) {
            const uint32_t h = wave[k];
            Hit & hit = out[where[h].first][where[h].second];
            const TbRegion & rg = regions[h];
            hit.has_cigar = true;
            if( scores_from_regions )
                hit.score = rg.fwd_score;
            if( rg.status != 0 ) {
                // no positive cell: the reference leaves the region undefined here
                hit.q_start = hit.q_end = hit.d_start = hit.d_end = 0;
                hit.cigar.clear();
                continue;
            }
            hit.q_start = (uint32_t) rg.a_begin;
            hit.q_end = (uint32_t) rg.a_end;
            hit.d_start = (uint32_t) rg.b_begin;
            hit.d_end = (uint32_t) rg.b_end;
            // run-length encode the moves in alignment order; counts of 1 are
            // omitted (reference: src/algo/cigar.c:221-263)
            const char * mv = ops.data() + wops[k];
            uint32_t n = (uint32_t) std::min<uint64_t>( ops_len[k], wops[k + 1] - wops[k] );
            std::string cig;
            uint32_t i = n;
            char buf[24];
            while( i > 0 ) {
                const char op = mv[i - 1];
                uint32_t run = 0;
                while( i > 0 && mv[i - 1] == op ) {
                    run++;
                    i--;
                }
                if( run > 1 ) {
                    snprintf( buf, sizeof(buf), "%u", run );
                    cig += buf;
                }
                cig += op;
            }
            hit.cigar = std::move( cig );
        }
    }
    // a very large direction buffer (long pairs) is not kept for later calls,
    // whose scores, lists and database segments need the device memory
    if( d_tb_dirs_.bytes > ((uint64_t) 8 << 30) )
        d_tb_dirs_.release();
    if( timing ) {
        uint64_t max_cells = 0;
        uint32_t max_a = 0, max_b = 0;
        for( uint32_t h = 0; h < nh; h++ ) {
            const uint64_t A = h_qlen_[hits[h].qslot], B = db_.len[hits[h].id];
            if( A * B > max_cells ) {
                max_cells = A * B;
                max_a = (uint32_t) A;
                max_b = (uint32_t) B;
            }
        }
        if( fused )
            fprintf( stderr, "[ssa timing] traceback %u hits: forward with directions %.3f ms, reverse and walk "
                    "%.3f ms in %zu wave(s) (%.3f GB of directions); largest hit %u x %u\n", nh, t_dir, t_walk,
                    waves.size(), total_dir * 1e-9, max_a, max_b );
        else
            fprintf( stderr, "[ssa timing] traceback %u hits: forward %.3f ms, reverse %.3f ms, directions %.3f ms, "
                    "walk %.3f ms in %zu wave(s) (%.3f GB of directions); largest hit %u x %u\n", nh, t_fwd, t_rev,
                    t_dir, t_walk, waves.size(), total_dir * 1e-9, max_a, max_b );
    }
}

// Device memory for the direction words of one traceback wave: the setting of
// ssa_b200_set_traceback_memory, else the free device memory (plus what the
// direction buffer holds already) less a reserve.
uint64_t Engine::traceback_budget() {
    if( tb_budget_ )
        return tb_budget_;
    size_t free_b = 0, total_b = 0;
    CUDA_CHECK( cudaMemGetInfo( &free_b, &total_b ) );
    const uint64_t avail = (uint64_t) free_b + d_tb_dirs_.bytes;
    const uint64_t reserve = std::max<uint64_t>( (uint64_t) 4 << 30, (uint64_t) total_b / 16 );
    const uint64_t floor = (uint64_t) 256 << 20;
    return avail > reserve + floor ? avail - reserve : floor;
}

// ---- long pairs -------------------------------------------------------------------
// Query i against database unit units[i] alone: what sw_align / nw_align return
// for the query against a database holding only that sequence (one hit, or
// none for an empty sequence).  One warp scores each pair exactly
// (pair_kernel.cu); the hits then go through the traceback like a search's.
void Engine::align_pairs( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & units, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    const HostDb & db = database();
    serving_ = false;
    serve_layout_ = false;      // the query buffers are reused for this batch
    const uint32_t n = (uint32_t) queries.size();
    out.assign( n, {} );
    if( n == 0 )
        return;
    if( units.size() != n )
        fatal( "Internal error: pairs without a database sequence." );
    const int64_t mabs = max_abs_step( req );
    std::vector<uint32_t> work;     // pairs with a non-empty sequence, largest first
    uint32_t max_b = 0, max_a = 0;
    for( uint32_t i = 0; i < n; i++ ) {
        if( units[i] >= db.n_ids )
            fatal( "Internal error: database unit %u out of range.", units[i] );
        const uint32_t A = queries[i].len, B = db.len[units[i]];
        if( (int64_t) (A + B + 4) * (mabs + 1) * 2 > INT32_MAX )
            fatal( "Alignment of %u x %u residues exceeds the supported score range.", A, B );
        stats.cells += (uint64_t) A * B;
        if( B == 0 )
            continue;       // the reference never searches an empty sequence
        work.push_back( i );
        max_b = std::max( max_b, B );
        max_a = std::max( max_a, A );
    }
    std::stable_sort( work.begin(), work.end(), [&]( uint32_t x, uint32_t y ) {
        return (uint64_t) queries[x].len * db.len[units[x]] > (uint64_t) queries[y].len * db.len[units[y]];
    } );
    const bool timing = getenv( "SSA_B200_TIMING" ) != nullptr;
    CUDA_CHECK( cudaEventRecord( ev0_, stream_ ) );
    d_matrix_.ensure( 1024 * sizeof(int64_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_matrix_.p, req.matrix, 1024 * sizeof(int64_t), cudaMemcpyHostToDevice, stream_ ) );
    upload_queries( queries.data(), n, false, stats );
    d_counts_.ensure( 32 * sizeof(unsigned long long) );
    CUDA_CHECK( cudaMemsetAsync( d_counts_.p, 0, 32 * sizeof(unsigned long long), stream_ ) );
    const uint32_t nw = (uint32_t) work.size();
    // With alignments the traceback passes compute the score themselves: the
    // direction pass ends on cell (A - 1, B - 1) of the same recurrence
    // (Needleman-Wunsch), the forward region pass finds the same maximum when
    // the score table is symmetric (Smith-Waterman; it scores [query][db])
    bool symmetric = true;
    for( int d = 0; d < 32; d++ )
        for( int q = 0; q < 32; q++ )
            symmetric = symmetric && req.matrix[(d << 5) + q] == req.matrix[(q << 5) + d];
    const bool scores_in_traceback = req.align_type == COMPUTE_ALIGNMENT && (req.algo == 1 || symmetric);
    if( nw && scores_in_traceback ) {
        for( uint32_t k = 0; k < nw; k++ ) {
            const uint32_t i = work[k];
            Hit h;
            h.unit = units[i];
            h.id = units[i] / db.upi;
            out[i].push_back( h );
        }
    }
    else if( nw ) {
        std::vector<uint32_t> hs( nw ), hu( nw );
        for( uint32_t k = 0; k < nw; k++ ) {
            hs[k] = work[k];
            hu[k] = units[work[k]];
        }
        PairScoreParams p{};
        if( streaming_ ) {
            // the pairs' sequences gathered into a view of their own
            std::vector<uint32_t> ids;
            std::unordered_map<uint32_t, uint32_t> index;
            for( uint32_t & u : hu ) {
                auto it = index.find( u );
                if( it == index.end() ) {
                    it = index.emplace( u, (uint32_t) ids.size() ).first;
                    ids.push_back( u );
                }
                u = it->second;
            }
            p.db = gather_view( ids, stats );
        }
        else {
            p.db = db_view();
        }
        p.qcodes = d_qcodes_.as<uint8_t>();
        p.qoff = d_qoff_.as<uint64_t>();
        p.qlen = d_qlen_.as<uint32_t>();
        p.pair_slot = (const uint32_t *) d_pair_slot_.ensure( nw * sizeof(uint32_t) );
        p.pair_unit = (const uint32_t *) d_pair_unit_.ensure( nw * sizeof(uint32_t) );
        p.n_pairs = nw;
        p.matrix = d_matrix_.as<int64_t>();
        p.gap_open = req.gap_open;
        p.gap_extend = req.gap_extend;
        p.score = (int32_t *) d_pair_score_.ensure( nw * sizeof(int32_t) );
        p.counter = d_counts_.as<unsigned long long>() + 15;      // bytes 120..127
        p.error_flags = d_counts_.as<unsigned>() + 2;
        int per_sm = 0;
        CUDA_CHECK( launch_pair_score( req.algo, p, 0, stream_, &per_sm ) );
        const int grid = sms_ * std::max( 1, per_sm );
        if( max_a > (uint32_t) (32 * PAIR_R) ) {
            p.scratch_cols = max_b;
            p.scratch = (int4 *) d_scratch_.ensure( (size_t) grid * (PAIR_THREADS / (32 * PAIR_W)) * max_b * sizeof(int4) );
        }
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.pair_slot, hs.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice,
                stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( (void *) p.pair_unit, hu.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice,
                stream_ ) );
        stats.h2d_bytes += 2 * nw * sizeof(uint32_t);
        CUDA_CHECK( cudaEventRecord( ev_phase_[0], stream_ ) );
        CUDA_CHECK( launch_pair_score( req.algo, p, grid, stream_, nullptr ) );
        launches_++;
        CUDA_CHECK( cudaEventRecord( ev_phase_[1], stream_ ) );
        std::vector<int32_t> sc( nw );
        unsigned err = 0;
        CUDA_CHECK( cudaMemcpyAsync( sc.data(), p.score, nw * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaMemcpyAsync( &err, p.error_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        if( err )
            fatal( "Internal error in the GPU pair scores (flags 0x%x).", err );
        stats.d2h_bytes += nw * sizeof(int32_t);
        float ms = 0;
        CUDA_CHECK( cudaEventElapsedTime( &ms, ev_phase_[0], ev_phase_[1] ) );
        stats.entry_seconds += ms * 1e-3;
        stats.kernel_seconds += ms * 1e-3;
        if( timing )
            fprintf( stderr, "[ssa timing] pair scores: %u pairs, %.3f ms\n", nw, ms );
        for( uint32_t k = 0; k < nw; k++ ) {
            const uint32_t i = work[k];
            Hit h;
            h.score = sc[k];
            h.unit = units[i];
            h.id = units[i] / db.upi;
            h.q_index = 0;
            out[i].push_back( h );
        }
    }
    if( req.align_type == COMPUTE_ALIGNMENT && nw ) {
        std::vector<std::pair<uint32_t, uint32_t>> lists;
        for( uint32_t i = 0; i < n; i++ )
            if( !out[i].empty() )
                lists.emplace_back( i, i );
        const auto t0 = std::chrono::steady_clock::now();
        traceback( req, out, lists, stats, scores_in_traceback );
        stats.kernel_seconds += std::chrono::duration<double>( std::chrono::steady_clock::now() - t0 ).count();
    }
    CUDA_CHECK( cudaEventRecord( ev1_, stream_ ) );
    CUDA_CHECK( cudaEventSynchronize( ev1_ ) );
    float ms = 0;
    CUDA_CHECK( cudaEventElapsedTime( &ms, ev0_, ev1_ ) );
    stats.seconds_gpu += ms * 1e-3;
    stats.kernel_launches = launches_.load();
}

// ---- serving -------------------------------------------------------------------
// A server keeps a fixed number of query slots resident: slot s owns the codes at
// s * SERVE_QSTRIDE, its int32 profile at s * 32 * SERVE_MAX_QUERY and the score
// row s of d_serve_score_.  Each wave runs the entry pass and the cascade of every
// occupied slot over one segment of the length-sorted database; a slot that has
// seen every segment is finished (score rows to the host, schedule replay, heap,
// traceback) and freed for the next request.
constexpr uint32_t SERVE_QSTRIDE = SERVE_MAX_QUERY + 16;

// ---- database-sharded searches (one process per GPU, contiguous record
// ranges; the per-record results are gathered to one replaying process) ----
void Engine::shard_scores( const SearchRequest & req, const std::vector<QueryCodes> & queries, uint32_t id_lo,
        uint32_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16, SearchStats & stats ) {
    init_device();
    const HostDb & db = database();
    if( db.upi != 1 )
        fatal( "Database-sharded searches support one database strand." );
    if( streaming_ )
        fatal( "Database-sharded searches need the database resident on the device." );
    serving_ = false;
    serve_layout_ = false;
    last_shapes_.clear();
    id_hi = std::min( id_hi, db.n_ids );
    id_lo = std::min( id_lo, id_hi );
    const uint64_t width = id_hi - id_lo;
    const uint32_t nq_all = (uint32_t) queries.size();
    for( uint64_t k = 0; k < (uint64_t) nq_all * width; k++ ) {
        scores[k] = 0;
        blocks_entry[k] = -1;
        blocks_16[k] = -1;
    }
    if( width == 0 || queries.empty() )
        return;
    // this shard's non-empty records, longest first: the entry passes see it as
    // their whole database
    std::vector<uint32_t> shard;
    for( uint32_t id : db.order_desc )
        if( id >= id_lo && id < id_hi )
            shard.push_back( id );
    const uint64_t n_sh = shard.size();
    {
        uint32_t qmax = 0;
        for( const QueryCodes & q : queries )
            qmax = std::max( qmax, q.len );
        wide_ = needs_int64( req, qmax, db.max_len );
    }
    d_matrix_.ensure( 1024 * sizeof(int64_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_matrix_.p, req.matrix, 1024 * sizeof(int64_t), cudaMemcpyHostToDevice, stream_ ) );
    std::vector<uint32_t> full_order;
    full_order.swap( db_.order_desc );
    db_.order_desc = shard;
    if( n_sh )
        CUDA_CHECK( cudaMemcpyAsync( d_order_.p, shard.data(), n_sh * sizeof(uint32_t), cudaMemcpyHostToDevice,
                stream_ ) );
    const uint64_t pair_budget = this->pair_budget();
    const uint32_t batch = (uint32_t) std::max<uint64_t>( 1, std::min<uint64_t>( nq_all,
            pair_budget / std::max<uint64_t>( 1, db.n_ids ) ) );
    for( uint32_t b0 = 0; b0 < nq_all && n_sh; b0 += batch ) {
        const uint32_t nq = std::min( batch, nq_all - b0 );
        upload_queries( queries.data() + b0, nq, true, stats );
        for( uint32_t q = 0; q < nq; q++ ) {
            uint64_t res = 0;
            for( uint32_t id : shard )
                res += db.len[id];
            stats.cells += (uint64_t) h_qlen_[q] * res;
        }
        const size_t score_bytes = (size_t) nq * db.n_ids * sizeof(int32_t);
        d_score_.ensure( std::max<size_t>( score_bytes, 4 ) );
        if( wide_ )
            d_score64_.ensure( std::max<size_t>( 2 * score_bytes, 8 ) );
        const uint32_t cap = (uint32_t) std::min<uint64_t>( std::max<uint64_t>( (uint64_t) nq * n_sh, 1 ),
                0xffffffffull );
        d_list_a_.ensure( (size_t) cap * sizeof(PairTask) );
        d_list_b_.ensure( (size_t) cap * sizeof(PairTask) );
        d_counts_.ensure( 32 * sizeof(unsigned long long) );
        CUDA_CHECK( cudaMemsetAsync( d_counts_.p, 0, 32 * sizeof(unsigned long long), stream_ ) );
        unsigned * cnt = d_counts_.as<unsigned>();
        const int entry = req.bit_width;
        CUDA_CHECK( cudaEventRecord( ev_seg_[0], stream_ ) );
        if( fast_eligible( req ) || nw_fast_eligible( req ) )
            run_qpair_entry( req, nq, d_list_a_.as<PairTask>(), cnt + 0, cap, nullptr, 0, (uint32_t) n_sh );
        else
            run_pass( req.algo, entry, req, nq, nullptr, (uint64_t) nq * n_sh, true, d_list_a_.as<PairTask>(),
                    cnt + 0, cap );
        CUDA_CHECK( cudaEventRecord( ev_seg_[1], stream_ ) );
        std::vector<PairTask> list_entry, list_16;
        unsigned sa = 0, sb = 0;
        if( entry != 64 ) {
            CUDA_CHECK( cudaMemcpyAsync( &sa, cnt + 0, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
            CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
            sa = std::min( sa, cap );
            if( sa ) {
                const int w2 = (entry == 8) ? 16 : 64;
                PairTask * nx = (w2 == 16) ? d_list_b_.as<PairTask>() : nullptr;
                run_pass( req.algo, w2, req, nq, d_list_a_.as<PairTask>(), sa, false, nx, cnt + 1, cap );
                if( w2 == 16 ) {
                    CUDA_CHECK( cudaMemcpyAsync( &sb, cnt + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
                    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
                    sb = std::min( sb, cap );
                    if( sb )
                        run_pass( req.algo, 64, req, nq, d_list_b_.as<PairTask>(), sb, false, nullptr, cnt + 3, 0 );
                }
                list_entry.resize( sa );
                CUDA_CHECK( cudaMemcpyAsync( list_entry.data(), d_list_a_.p, sa * sizeof(PairTask),
                        cudaMemcpyDeviceToHost, stream_ ) );
                if( sb ) {
                    list_16.resize( sb );
                    CUDA_CHECK( cudaMemcpyAsync( list_16.data(), d_list_b_.p, sb * sizeof(PairTask),
                            cudaMemcpyDeviceToHost, stream_ ) );
                }
            }
        }
        int32_t * hs = (int32_t *) h_score_.ensure( std::max<size_t>( score_bytes, 4 ) );
        CUDA_CHECK( cudaMemcpyAsync( hs, d_score_.p, score_bytes, cudaMemcpyDeviceToHost, stream_ ) );
        int64_t * hs64 = nullptr;
        if( wide_ ) {
            hs64 = (int64_t *) h_score64_.ensure( 2 * score_bytes );
            CUDA_CHECK( cudaMemcpyAsync( hs64, d_score64_.p, 2 * score_bytes, cudaMemcpyDeviceToHost, stream_ ) );
        }
        unsigned err = 0;
        CUDA_CHECK( cudaMemcpyAsync( &err, cnt + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        if( err )
            fatal( "Internal error in the GPU search (flags 0x%x).", err );
        float ms = 0;
        CUDA_CHECK( cudaEventElapsedTime( &ms, ev_seg_[0], ev_seg_[1] ) );
        stats.entry_seconds += ms * 1e-3;
        stats.d2h_bytes += score_bytes + (sa + sb) * sizeof(PairTask);
        for( uint32_t q = 0; q < nq; q++ ) {
            const uint64_t row = (uint64_t) (b0 + q) * width;
            ReplayQuery rq;
            rq.score = hs + (size_t) q * db.n_ids;
            rq.score64 = hs64 ? hs64 + (size_t) q * db.n_ids : nullptr;
            for( uint32_t id : shard )
                scores[row + (id - id_lo)] = rq.score_of( id );
        }
        for( const PairTask & t : list_entry )
            blocks_entry[(uint64_t) (b0 + t.qslot) * width + (t.id - id_lo)] = t.nb_prev;
        for( const PairTask & t : list_16 )
            blocks_16[(uint64_t) (b0 + t.qslot) * width + (t.id - id_lo)] = t.nb_prev;
    }
    db_.order_desc.swap( full_order );
    if( !db_.order_desc.empty() )
        CUDA_CHECK( cudaMemcpyAsync( d_order_.p, db_.order_desc.data(), db_.order_desc.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
    stats.kernel_launches = launches_.load();
}

void Engine::align_hits( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    init_device();
    database();
    serving_ = false;
    serve_layout_ = false;
    d_matrix_.ensure( 1024 * sizeof(int64_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_matrix_.p, req.matrix, 1024 * sizeof(int64_t), cudaMemcpyHostToDevice, stream_ ) );
    const uint32_t nq = (uint32_t) queries.size();
    const uint32_t batch = 65535;
    for( uint32_t b0 = 0; b0 < nq; b0 += batch ) {
        const uint32_t n = std::min( batch, nq - b0 );
        upload_queries( queries.data() + b0, n, false, stats );
        std::vector<std::pair<uint32_t, uint32_t>> lists;
        for( uint32_t q = 0; q < n; q++ )
            lists.emplace_back( b0 + q, q );
        traceback( req, out, lists, stats );
    }
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
}

void Engine::serve_restore( const SearchRequest & req ) {
    const uint32_t S = serve_slots_;
    d_matrix_.ensure( 1024 * sizeof(int64_t) );
    CUDA_CHECK( cudaMemcpyAsync( d_matrix_.p, req.matrix, 1024 * sizeof(int64_t), cudaMemcpyHostToDevice, stream_ ) );
    h_qoff_.assign( S, 0 );
    h_qlen_.assign( S, 0 );
    h_qpad_.assign( S, 256 );
    h_prof_off_.assign( S, 0 );
    for( uint32_t s = 0; s < S; s++ ) {
        const uint32_t len = (uint32_t) serve_codes_[s].size();
        h_qoff_[s] = (uint64_t) s * SERVE_QSTRIDE;
        h_qlen_[s] = len;
        h_qpad_[s] = std::max<uint32_t>( 256, (len + 255u) & ~255u );
        h_prof_off_[s] = (uint64_t) s * 32 * SERVE_MAX_QUERY;
    }
    d_qcodes_.ensure( (size_t) S * SERVE_QSTRIDE + 16 );
    d_qoff_.ensure( S * sizeof(uint64_t) );
    d_qlen_.ensure( S * sizeof(uint32_t) );
    d_qpad_.ensure( S * sizeof(uint32_t) );
    d_prof_off_.ensure( S * sizeof(uint64_t) );
    d_prof_.ensure( (size_t) S * 32 * SERVE_MAX_QUERY * sizeof(int32_t) );
    d_counts_.ensure( 32 * sizeof(unsigned long long) );
    CUDA_CHECK( cudaMemcpyAsync( d_qoff_.p, h_qoff_.data(), S * sizeof(uint64_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qlen_.p, h_qlen_.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qpad_.p, h_qpad_.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_prof_off_.p, h_prof_off_.data(), S * sizeof(uint64_t), cudaMemcpyHostToDevice,
            stream_ ) );
    for( uint32_t s = 0; s < S; s++ )
        if( !serve_codes_[s].empty() )
            CUDA_CHECK( cudaMemcpyAsync( d_qcodes_.as<uint8_t>() + h_qoff_[s], serve_codes_[s].data(),
                    serve_codes_[s].size(), cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
    prof_width_ = -1;
    serve_layout_ = true;
}

std::vector<uint32_t> Engine::serve_open( const SearchRequest & req, uint32_t slots, uint32_t segments ) {
    init_device();
    const HostDb & db = database();
    if( needs_int64( req, SERVE_MAX_QUERY, db.max_len ) )
        fatal( "The server scores in int32: the score table and gap penalties can exceed that range on this "
               "database; use sw_align/nw_align." );
    wide_ = false;
    serve_slots_ = slots;
    serve_codes_.assign( slots, {} );
    d_serve_score_.ensure( std::max<size_t>( 4, (size_t) slots * db.n_ids * sizeof(int32_t) ) );
    serve_layout_ = false;
    serve_restore( req );
    // the query-independent lane schedule of the entry width, computed once here
    // rather than in the first request's latency
    if( req.bit_width != 64 )
        ranks( req.chunk_size, req.bit_width == 8 ? req.lanes8 : req.lanes16 );
    // segments of the length-sorted sequences holding about equal residues
    const uint32_t n = (uint32_t) db.order_desc.size();
    segments = std::max<uint32_t>( 1, std::min<uint32_t>( segments, std::max<uint32_t>( 1, n ) ) );
    std::vector<uint32_t> bounds{ 0 };
    uint64_t acc = 0;
    for( uint32_t i = 0; i < n && bounds.size() < segments; i++ ) {
        acc += db.len[db.order_desc[i]];
        if( acc * segments >= db.residues * (uint64_t) bounds.size() )
            bounds.push_back( i + 1 );
    }
    if( bounds.back() != n )
        bounds.push_back( n );
    return bounds;
}

void Engine::serve_load( uint32_t slot, const uint8_t * codes, uint32_t len ) {
    serve_codes_[slot].assign( codes, codes + len );
    if( !serve_layout_ )
        return;     // restored before the next wave
    h_qlen_[slot] = len;
    h_qpad_[slot] = std::max<uint32_t>( 256, (len + 255u) & ~255u );
    CUDA_CHECK( cudaMemcpyAsync( d_qcodes_.as<uint8_t>() + h_qoff_[slot], codes, len, cudaMemcpyHostToDevice,
            stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qlen_.as<uint32_t>() + slot, &h_qlen_[slot], sizeof(uint32_t),
            cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaMemcpyAsync( d_qpad_.as<uint32_t>() + slot, &h_qpad_[slot], sizeof(uint32_t),
            cudaMemcpyHostToDevice, stream_ ) );
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
    prof_width_ = -1;
}

void Engine::serve_wave( const SearchRequest & req, const std::vector<uint32_t> & active, uint32_t seq_lo,
        uint32_t seq_hi, std::vector<PairTask> & ovf_entry, std::vector<PairTask> & ovf16, SearchStats & stats ) {
    ovf_entry.clear();
    ovf16.clear();
    if( active.empty() || seq_hi <= seq_lo )
        return;
    if( !serve_layout_ )
        serve_restore( req );
    serving_ = true;
    wide_ = false;                 // the server's settings were checked at serve_open
    const uint32_t n_seg = seq_hi - seq_lo;
    max_qlen_ = 0;
    uint64_t seg_res = 0;
    for( uint32_t i = seq_lo; i < seq_hi; i++ )
        seg_res += db_.len[db_.order_desc[i]];
    for( uint32_t s : active ) {
        max_qlen_ = std::max( max_qlen_, h_qlen_[s] );
        stats.cells += (uint64_t) h_qlen_[s] * seg_res;
    }
    const uint64_t n_pairs = (uint64_t) active.size() * n_seg;
    const uint32_t cap = (uint32_t) std::min<uint64_t>( std::max<uint64_t>( n_pairs, 1 ), 0xffffffffull );
    d_list_a_.ensure( (size_t) cap * sizeof(PairTask) );
    d_list_b_.ensure( (size_t) cap * sizeof(PairTask) );
    CUDA_CHECK( cudaMemsetAsync( d_counts_.p, 0, 32 * sizeof(unsigned long long), stream_ ) );
    unsigned * cnt = d_counts_.as<unsigned>();
    const int entry = req.bit_width;
    CUDA_CHECK( cudaEventRecord( ev_phase_[0], stream_ ) );
    if( fast_eligible( req ) || nw_fast_eligible( req ) ) {
        run_qpair_entry( req, serve_slots_, d_list_a_.as<PairTask>(), cnt + 0, cap, &active, seq_lo, seq_hi );
    }
    else {
        d_slots_.ensure( active.size() * sizeof(uint32_t) );
        CUDA_CHECK( cudaMemcpyAsync( d_slots_.p, active.data(), active.size() * sizeof(uint32_t),
                cudaMemcpyHostToDevice, stream_ ) );
        run_pass( req.algo, entry, req, serve_slots_, nullptr, n_pairs, true, d_list_a_.as<PairTask>(), cnt + 0, cap,
                d_slots_.as<uint32_t>(), (uint32_t) active.size(), seq_lo );
    }
    CUDA_CHECK( cudaEventRecord( ev_phase_[1], stream_ ) );
    unsigned n_a = 0, n_b = 0;
    if( entry != 64 ) {
        CUDA_CHECK( cudaMemcpyAsync( &n_a, cnt + 0, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
        CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
        n_a = std::min( n_a, cap );
        if( n_a ) {
            const int w2 = (entry == 8) ? 16 : 64;
            PairTask * nx = (w2 == 16) ? d_list_b_.as<PairTask>() : nullptr;
            run_pass( req.algo, w2, req, serve_slots_, d_list_a_.as<PairTask>(), n_a, false, nx, cnt + 1, cap );
            if( w2 == 16 ) {
                CUDA_CHECK( cudaMemcpyAsync( &n_b, cnt + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
                CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
                n_b = std::min( n_b, cap );
                if( n_b )
                    run_pass( req.algo, 64, req, serve_slots_, d_list_b_.as<PairTask>(), n_b, false, nullptr, cnt + 3,
                            0 );
            }
            ovf_entry.resize( n_a );
            CUDA_CHECK( cudaMemcpyAsync( ovf_entry.data(), d_list_a_.p, n_a * sizeof(PairTask),
                    cudaMemcpyDeviceToHost, stream_ ) );
            if( n_b ) {
                ovf16.resize( n_b );
                CUDA_CHECK( cudaMemcpyAsync( ovf16.data(), d_list_b_.p, n_b * sizeof(PairTask),
                        cudaMemcpyDeviceToHost, stream_ ) );
            }
        }
    }
    unsigned err = 0;
    CUDA_CHECK( cudaMemcpyAsync( &err, cnt + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_ ) );
    CUDA_CHECK( cudaEventRecord( ev_phase_[2], stream_ ) );
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
    serving_ = false;
    if( err )
        fatal( "Internal error in the GPU search (flags 0x%x).", err );
    float ms[2];
    CUDA_CHECK( cudaEventElapsedTime( &ms[0], ev_phase_[0], ev_phase_[1] ) );
    CUDA_CHECK( cudaEventElapsedTime( &ms[1], ev_phase_[1], ev_phase_[2] ) );
    stats.entry_seconds += ms[0] * 1e-3;
    stats.kernel_seconds += (ms[0] + ms[1]) * 1e-3;
    stats.overflow8 += n_a;
    stats.overflow16 += n_b;
}

void Engine::serve_finish( const SearchRequest & req, const std::vector<uint32_t> & done,
        std::vector<ReplayQuery> & rq, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    out.assign( serve_slots_, {} );
    if( done.empty() )
        return;
    if( !serve_layout_ )
        serve_restore( req );
    const uint32_t nd = (uint32_t) done.size();
    const size_t row = (size_t) db_.n_ids;
    int32_t * hs = (int32_t *) h_score_.ensure( std::max<size_t>( 4, nd * row * sizeof(int32_t) ) );
    for( uint32_t i = 0; i < nd; i++ )
        CUDA_CHECK( cudaMemcpyAsync( hs + i * row, d_serve_score_.as<int32_t>() + (size_t) done[i] * row,
                row * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_ ) );
    CUDA_CHECK( cudaStreamSynchronize( stream_ ) );
    stats.d2h_bytes += nd * row * sizeof(int32_t);
    const int entry = req.bit_width;
    const uint32_t * rank_entry =
            (entry == 64) ? nullptr : ranks( req.chunk_size, entry == 8 ? req.lanes8 : req.lanes16 );
    {
        std::atomic<uint32_t> next{ 0 };
        std::vector<ReplayCounts> counts( nd );
        auto work = [&]() {
            for( ;; ) {
                const uint32_t i = next.fetch_add( 1 );
                if( i >= nd )
                    break;
                rq[i].score = hs + i * row;
                std::sort( rq[i].ovf_entry.begin(), rq[i].ovf_entry.end() );
                std::sort( rq[i].ovf16.begin(), rq[i].ovf16.end() );
                replay_query( db_, req, rq[i], rank_entry, out[done[i]], counts[i] );
            }
        };
        const unsigned nthreads = std::min<unsigned>( std::max( 1u, std::thread::hardware_concurrency() ), nd );
        std::vector<std::thread> th;
        for( unsigned k = 1; k < nthreads; k++ )
            th.emplace_back( work );
        work();
        for( auto & t : th )
            t.join();
    }
    if( req.align_type == COMPUTE_ALIGNMENT ) {
        max_qlen_ = 0;
        for( uint32_t s : done )
            max_qlen_ = std::max( max_qlen_, h_qlen_[s] );
        std::vector<std::pair<uint32_t, uint32_t>> lists;
        for( uint32_t sl : done )
            lists.emplace_back( sl, sl );
        traceback( req, out, lists, stats );
    }
}

// ---- free functions ------------------------------------------------------------
// One engine per process; the search entry points and a server's waves take
// turns on it.
static std::mutex g_engine_mutex;

void engine_search( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & groups, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().search( req, queries, groups, out, stats );
}

void engine_align_pairs( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        const std::vector<uint32_t> & units, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().align_pairs( req, queries, units, out, stats );
}

void engine_set_traceback_memory( uint64_t bytes ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().set_traceback_budget( bytes );
}

void engine_set_db_memory( uint64_t bytes ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().set_db_budget( bytes );
}

bool engine_streaming() {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine & e = Engine::get();
    e.database();
    return e.streaming();
}

const HostDb & engine_database() {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    return Engine::get().database();
}

void engine_invalidate_database() {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().invalidate();
}

void engine_shutdown() {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().shutdown();
}

std::vector<uint32_t> engine_serve_open( const SearchRequest & req, uint32_t slots, uint32_t segments ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    return Engine::get().serve_open( req, slots, segments );
}

void engine_serve_load( uint32_t slot, const uint8_t * codes, uint32_t len ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().serve_load( slot, codes, len );
}

void engine_serve_wave( const SearchRequest & req, const std::vector<uint32_t> & active, uint32_t seq_lo,
        uint32_t seq_hi, std::vector<ServeOverflow> & ovf_entry, std::vector<ServeOverflow> & ovf16,
        SearchStats & stats ) {
    std::vector<PairTask> a, b;
    {
        std::lock_guard<std::mutex> lock( g_engine_mutex );
        Engine::get().serve_wave( req, active, seq_lo, seq_hi, a, b, stats );
    }
    ovf_entry.clear();
    ovf16.clear();
    for( const PairTask & t : a )
        ovf_entry.push_back( ServeOverflow{ t.qslot, t.id, t.nb_prev } );
    for( const PairTask & t : b )
        ovf16.push_back( ServeOverflow{ t.qslot, t.id, t.nb_prev } );
}

void engine_serve_finish( const SearchRequest & req, const std::vector<uint32_t> & done,
        std::vector<ReplayQuery> & rq, std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().serve_finish( req, done, rq, out, stats );
}

void engine_shard_scores( const SearchRequest & req, const std::vector<QueryCodes> & queries, uint32_t id_lo,
        uint32_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16, SearchStats & stats ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().shard_scores( req, queries, id_lo, id_hi, scores, blocks_entry, blocks_16, stats );
}

void engine_align_hits( const SearchRequest & req, const std::vector<QueryCodes> & queries,
        std::vector<std::vector<Hit>> & out, SearchStats & stats ) {
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    Engine::get().align_hits( req, queries, out, stats );
}

// Host-only: the database's record lengths through the plugin (no device),
// as the schedule replay needs them.
void lengths_db( HostDb & db ) {
    db = HostDb();
    const size_t n = ssa_db_get_sequence_count();
    if( n > UINT32_MAX )
        fatal( "Database has %zu sequences; at most %u are supported.", n, UINT32_MAX );
    db.n_ids = db.n_records = (uint32_t) n;
    db.upi = 1;
    db.len.assign( n, 0 );
    for( size_t id = 0; id < n; id++ ) {
        p_seqinfo info = ssa_db_get_sequence( id );
        if( !info )
            fatal( "Could not get sequence from DB: %zu", id );
        db.len[id] = (uint32_t) info->seqlen;
        db.max_len = std::max( db.max_len, db.len[id] );
        db.residues += info->seqlen;
    }
    db.nonempty_before.assign( n + 1, 0 );
    for( uint32_t id = 0; id < db.n_ids; id++ ) {
        db.nonempty_before[id + 1] = db.nonempty_before[id] + (db.len[id] ? 1 : 0);
        if( db.len[id] )
            db.order_desc.push_back( id );
    }
    std::stable_sort( db.order_desc.begin(), db.order_desc.end(),
            [&]( uint32_t a, uint32_t b ) { return db.len[a] > db.len[b]; } );
    db.mean_len = db.order_desc.empty() ? 0.0 : (double) db.residues / (double) db.order_desc.size();
}

std::string tuning_report() {
    const TuningTable & t = tuning();
    std::string out = "{\"source\": \"";
    for( char c : t.source )
        if( c != '"' && c != '\\' )
            out += c;
    out += "\", \"version\": " + std::to_string( t.version ) + ", \"device\": \"";
    for( char c : t.device )
        if( c != '"' && c != '\\' )
            out += c;
    out += "\", \"last_call\": [";
    std::lock_guard<std::mutex> lock( g_engine_mutex );
    bool first = true;
    for( const auto & u : Engine::get().last_shapes_ ) {
        char buf[160];
        const bool qp = strncmp( u.kernel, "sw_fast", 7 ) != 0;
        snprintf( buf, sizeof buf, "%s{\"kernel\": \"%s\", \"%s\": %d, \"%s\": %d, \"%s\": %u, \"bucket\": %d}",
                first ? "" : ", ", u.kernel, qp ? "R" : "G", u.a, qp ? "ctas_per_sm" : "R", u.b,
                qp ? "query_pairs" : "queries", u.n, u.bucket );
        out += buf;
        first = false;
    }
    out += "]}";
    return out;
}

uint64_t engine_kernel_launches() {
    return Engine::get().launches();
}

}  // namespace ssa
