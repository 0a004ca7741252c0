// replay.cpp -- reproduces the order in which the CPU library inserts scores
// into its top-hit heap, and the heap itself.
//
// The GPU computes every (query, sequence) score at once, but the CPU
// library's result set depends on insertion order whenever scores tie at the
// heap boundary: its min-heap replaces the root only on a strictly greater
// score (reference: src/util/minheap.c:50-91), so which of several tied
// sequences survive depends on when each arrived.  The arrival order is fixed
// by the database chunks (ID ranges of chunk_size records, empty records
// skipped; src/db_adapter.c:212-239), by the SIMD channel scheduler inside
// each chunk (a sequence enters the lowest free lane at a block where some
// lane finished, and reports at the first block after its last one;
// src/algo/simd/search_simd_sw.c:338-428), and by the overflow cascade, which
// inserts a chunk's 8-bit reports first, then its 16-bit re-run reports in
// their own schedule, then the 64-bit re-runs in order
// (src/algo/8/search_8.c:94-124, src/algo/16/search_16.c:92-114,
// src/algo/64/search_64.c:44-56).  This file replays exactly that, from the
// per-sequence scores and the block counts the GPU passes return.
#include "ssa_internal.h"

#include <algorithm>
#include <cstring>
#include <tuple>

namespace ssa {

// Report order of a list of sequences scheduled on `lanes` channels, where
// sequence k occupies nb[k] blocks.  Returns indices into the list.
static void simulate_lanes( int lanes, const std::vector<int32_t> & nb, std::vector<uint32_t> & order ) {
    const size_t n = nb.size();
    order.clear();
    if( n == 0 )
        return;
    // free time of each lane; a lane that frees at block t takes the next
    // sequence in lane order among all lanes freeing at t
    std::vector<int64_t> free_at( (size_t) lanes, 0 );
    std::vector<std::tuple<int64_t, int, uint32_t>> ends;
    ends.reserve( n );
    for( size_t k = 0; k < n; k++ ) {
        int best = 0;
        for( int c = 1; c < lanes; c++ )
            if( free_at[c] < free_at[best] )
                best = c;
        const int64_t t_end = free_at[best] + nb[k];
        ends.emplace_back( t_end, best, (uint32_t) k );
        free_at[best] = t_end;
    }
    std::sort( ends.begin(), ends.end() );
    order.resize( n );
    for( size_t k = 0; k < n; k++ )
        order[k] = std::get<2>( ends[k] );
}

void schedule_ranks( const HostDb & db, size_t chunk_size, int lanes, std::vector<uint32_t> & rank ) {
    rank.assign( db.n_ids, 0 );
    std::vector<uint32_t> ids;
    std::vector<int32_t> nb;
    std::vector<uint32_t> order;
    const uint64_t cs = (uint64_t) chunk_size * db.upi;    // a chunk of records, in units
    for( uint64_t start = 0; start < db.n_ids; start += cs ) {
        const uint64_t end = std::min<uint64_t>( db.n_ids, start + cs );
        ids.clear();
        nb.clear();
        for( uint64_t id = start; id < end; id++ ) {
            if( db.len[id] == 0 )
                continue;
            ids.push_back( (uint32_t) id );
            nb.push_back( (int32_t) ((db.len[id] + 3) / 4) );
        }
        simulate_lanes( lanes, nb, order );
        for( size_t k = 0; k < order.size(); k++ )
            rank[ids[order[k]]] = (uint32_t) k;
    }
}

namespace {

// Bit-identical restatement of the reference's fixed-size min-heap
// (reference: src/util/minheap.c:50-91).
struct MinHeap {
    struct Elem {
        uint32_t id;       // database unit
        int64_t score;
        uint32_t q = 0;    // query strand or frame
    };
    size_t alloc;
    std::vector<Elem> a;

    explicit MinHeap( size_t k ) : alloc( k ) { a.reserve( k ); }

    bool full() const { return a.size() >= alloc; }
    int64_t root() const { return a[0].score; }

    void add( uint32_t id, int64_t score, uint32_t q = 0 ) {
        if( alloc == 0 )
            return;
        Elem n{ id, score, q };
        if( a.size() < alloc ) {
            size_t i = a.size();
            a.push_back( n );
            while( i > 0 && n.score < a[(i - 1) / 2].score ) {
                a[i] = a[(i - 1) / 2];
                i = (i - 1) / 2;
            }
            a[i] = n;
        }
        else if( a[0].score < n.score ) {
            size_t p = 0, c = 1;
            const size_t count = a.size();
            while( c < count ) {
                if( c + 1 < count && a[c + 1].score < a[c].score )
                    c++;
                if( a[c].score < n.score )
                    a[p] = a[c];
                else
                    break;
                p = c;
                c = 2 * p + 1;
            }
            a[p] = n;
        }
    }
};

// (id, blocks) lists sorted by id, looked up per chunk.
struct BlockMap {
    const std::vector<std::pair<uint32_t, int32_t>> & v;
    size_t lower( uint32_t id ) const {
        return (size_t) (std::lower_bound( v.begin(), v.end(), std::make_pair( id, INT32_MIN ) ) - v.begin());
    }
    bool find( uint32_t id, int32_t & nb ) const {
        size_t k = lower( id );
        if( k < v.size() && v[k].first == id ) {
            nb = v[k].second;
            return true;
        }
        return false;
    }
};

}  // namespace

void replay_query( const HostDb & db, const SearchRequest & req, const ReplayQuery & rq, const uint32_t * rank_entry,
        std::vector<Hit> & hits, ReplayCounts & counts ) {
    MinHeap heap( req.hitcount );
    const size_t cs = (req.chunk_size ? req.chunk_size : 1000) * (size_t) db.upi;   // records -> units
    const int lanes_entry = req.bit_width == 8 ? req.lanes8 : req.lanes16;
    BlockMap ovfE{ rq.ovf_entry }, ovf16{ rq.ovf16 };

    std::vector<std::pair<uint32_t, uint32_t>> cand;   // (rank, id)
    std::vector<uint32_t> ids, order, order16, next, list64;
    std::vector<int32_t> nb;

    for( uint64_t start = 0; start < db.n_ids; start += cs ) {
        const uint64_t end = std::min<uint64_t>( db.n_ids, start + cs );
        // a chunk without non-empty records ends the search: the reference's
        // drivers loop while the chunk is non-empty (src/algo/8/search_8.c:652,
        // src/algo/16/search_16.c:785, src/algo/64/search_64.c:963)
        if( db.nonempty_before[end] == db.nonempty_before[start] )
            break;
        const bool has_ovf = req.bit_width != 64 && ovfE.lower( (uint32_t) start ) < rq.ovf_entry.size()
                && rq.ovf_entry[ovfE.lower( (uint32_t) start )].first < end;
        if( !has_ovf ) {
            // every sequence of the chunk reported at the entry pass: the
            // order is the query-independent schedule
            const bool filter = heap.full();
            const int64_t r = filter ? heap.root() : 0;
            cand.clear();
            for( uint64_t id = start; id < end; id++ ) {
                if( db.len[id] == 0 )
                    continue;
                const int64_t s = rq.score_of( id );
                if( filter && s <= r )
                    continue;
                cand.emplace_back( req.bit_width == 64 ? (uint32_t) (id - start) : rank_entry[id], (uint32_t) id );
            }
            if( cand.empty() )
                continue;
            std::sort( cand.begin(), cand.end() );
            for( auto & c : cand )
                heap.add( c.second, rq.score_of( c.second ) );
            continue;
        }
        // the chunk has overflowing sequences: re-run its schedules
        ids.clear();
        nb.clear();
        for( uint64_t id = start; id < end; id++ ) {
            if( db.len[id] == 0 )
                continue;
            int32_t b;
            if( !ovfE.find( (uint32_t) id, b ) )
                b = (int32_t) ((db.len[id] + 3) / 4);
            ids.push_back( (uint32_t) id );
            nb.push_back( b );
        }
        simulate_lanes( lanes_entry, nb, order );
        next.clear();
        const size_t n_entry_before = next.size();
        for( uint32_t k : order ) {
            const uint32_t id = ids[k];
            int32_t b;
            if( ovfE.find( id, b ) )
                next.push_back( id );
            else
                heap.add( id, rq.score_of( id ) );
        }
        if( req.bit_width == 8 )
            counts.overflow8 += next.size() - n_entry_before;
        else
            counts.overflow16 += next.size() - n_entry_before;
        if( req.bit_width == 8 && !next.empty() ) {
            nb.clear();
            for( uint32_t id : next ) {
                int32_t b;
                if( !ovf16.find( id, b ) )
                    b = (int32_t) ((db.len[id] + 3) / 4);
                nb.push_back( b );
            }
            simulate_lanes( req.lanes16, nb, order16 );
            list64.clear();
            for( uint32_t k : order16 ) {
                const uint32_t id = next[k];
                int32_t b;
                if( ovf16.find( id, b ) )
                    list64.push_back( id );
                else
                    heap.add( id, rq.score_of( id ) );
            }
            counts.overflow16 += list64.size();
            for( uint32_t id : list64 )
                heap.add( id, rq.score_of( id ) );
        }
        else {
            for( uint32_t id : next )
                heap.add( id, rq.score_of( id ) );
        }
    }

    // sort by score, then ID, both descending (reference: src/util/minheap.c:93-106)
    std::vector<MinHeap::Elem> e = heap.a;
    std::sort( e.begin(), e.end(), []( const MinHeap::Elem & x, const MinHeap::Elem & y ) {
        if( x.score != y.score )
            return x.score > y.score;
        return x.id > y.id;
    } );
    hits.clear();
    hits.resize( e.size() );
    for( size_t k = 0; k < e.size(); k++ ) {
        hits[k].score = e[k].score;
        hits[k].unit = e[k].id;
        hits[k].id = e[k].id / db.upi;
        hits[k].db_strand = (uint8_t) (e[k].id % db.upi);
    }
}

// A query searched as several sequences (strands, or translated frames): the
// reference runs every chunk once per query sequence into the same heap, then
// re-runs the chunk's overflow list, which holds the overflowing units of all
// query sequences in report order, at 16 bits for every query sequence, and its
// 16-bit overflow list at 64 bits for every query sequence
// (src/algo/8/search_8.c:94-124, src/algo/16/search_16.c:92-114,
// src/algo/64/search_64.c:44-56).  Every report carries the pair's exact
// score, which the GPU passes leave in the score rows.
void replay_frames( const HostDb & db, const SearchRequest & req, const ReplayQuery * rq, uint32_t F,
        std::vector<Hit> & hits, ReplayCounts & counts ) {
    MinHeap heap( req.hitcount );
    const size_t cs = (req.chunk_size ? req.chunk_size : 1000) * (size_t) db.upi;
    const int lanes_entry = req.bit_width == 8 ? req.lanes8 : req.lanes16;
    std::vector<BlockMap> ovfE, ovf16;
    for( uint32_t q = 0; q < F; q++ ) {
        ovfE.push_back( BlockMap{ rq[q].ovf_entry } );
        ovf16.push_back( BlockMap{ rq[q].ovf16 } );
    }
    auto blocks = [&]( uint32_t u ) { return (int32_t) ((db.len[u] + 3) / 4); };
    std::vector<uint32_t> units, order, ovf_chunk, list64;
    std::vector<int32_t> nb;
    for( uint64_t start = 0; start < db.n_ids; start += cs ) {
        const uint64_t end = std::min<uint64_t>( db.n_ids, start + cs );
        if( db.nonempty_before[end] == db.nonempty_before[start] )
            break;
        units.clear();
        for( uint64_t u = start; u < end; u++ )
            if( db.len[u] )
                units.push_back( (uint32_t) u );
        if( req.bit_width == 64 ) {
            for( uint32_t q = 0; q < F; q++ )
                for( uint32_t u : units )
                    heap.add( u, rq[q].score_of( u ), q );
            continue;
        }
        ovf_chunk.clear();
        for( uint32_t q = 0; q < F; q++ ) {
            nb.clear();
            for( uint32_t u : units ) {
                int32_t b;
                nb.push_back( ovfE[q].find( u, b ) ? b : blocks( u ) );
            }
            simulate_lanes( lanes_entry, nb, order );
            for( uint32_t k : order ) {
                const uint32_t u = units[k];
                int32_t b;
                if( ovfE[q].find( u, b ) )
                    ovf_chunk.push_back( u );
                else
                    heap.add( u, rq[q].score_of( u ), q );
            }
        }
        if( ovf_chunk.empty() )
            continue;
        if( req.bit_width == 8 ) {
            counts.overflow8 += ovf_chunk.size();
            list64.clear();
            for( uint32_t q = 0; q < F; q++ ) {
                // a pair that did not overflow at 8 bits reports at 16 bits too
                nb.clear();
                for( uint32_t u : ovf_chunk ) {
                    int32_t b8, b16;
                    nb.push_back( (ovfE[q].find( u, b8 ) && ovf16[q].find( u, b16 )) ? b16 : blocks( u ) );
                }
                simulate_lanes( req.lanes16, nb, order );
                for( uint32_t k : order ) {
                    const uint32_t u = ovf_chunk[k];
                    int32_t b8, b16;
                    if( ovfE[q].find( u, b8 ) && ovf16[q].find( u, b16 ) )
                        list64.push_back( u );
                    else
                        heap.add( u, rq[q].score_of( u ), q );
                }
            }
            counts.overflow16 += list64.size();
            for( uint32_t q = 0; q < F; q++ )
                for( uint32_t u : list64 )
                    heap.add( u, rq[q].score_of( u ), q );
        }
        else {
            counts.overflow16 += ovf_chunk.size();
            for( uint32_t q = 0; q < F; q++ )
                for( uint32_t u : ovf_chunk )
                    heap.add( u, rq[q].score_of( u ), q );
        }
    }
    // score, then database ID, both descending; entries equal in both keep
    // their heap order (the reference's qsort of the heap array is a stable
    // merge sort: src/util/minheap.c:93-106)
    std::vector<MinHeap::Elem> e = heap.a;
    std::stable_sort( e.begin(), e.end(), [&]( const MinHeap::Elem & x, const MinHeap::Elem & y ) {
        if( x.score != y.score )
            return x.score > y.score;
        return x.id / db.upi > y.id / db.upi;
    } );
    hits.clear();
    hits.resize( e.size() );
    for( size_t k = 0; k < e.size(); k++ ) {
        hits[k].score = e[k].score;
        hits[k].unit = e[k].id;
        hits[k].id = e[k].id / db.upi;
        hits[k].db_strand = (uint8_t) (e[k].id % db.upi);
        hits[k].q_index = e[k].q;
    }
}

}  // namespace ssa
