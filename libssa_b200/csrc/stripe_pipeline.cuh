// stripe_pipeline.cuh -- several warps on one alignment.
//
// A wavefront kernel cuts the query into stripes of 32 x R rows; one warp
// sweeps a stripe over all database columns (lane k on column s - k at step s)
// and hands its bottom row to the next stripe.  With one warp per alignment the
// largest alignment of a batch bounds the launch, because a warp's rows form a
// dependent chain.  Here a group of W warps shares an alignment: stripe i goes
// to warp i % W, and the group advances in steps of one chunk (32 wavefront
// steps) with a group barrier after each step.  Stripe i starts at least two
// steps after stripe i - 1 (four where it follows from the previous super-pass
// of W stripes), so every boundary column it reads was written in an earlier
// step:
//
//   * between the warps of one super-pass the bottom row travels through a
//     shared-memory ring of RING columns per warp, double-buffered by
//     super-pass parity (the producer runs at most 2 chunks = 64 columns ahead);
//   * from the last warp of a super-pass to warp 0 of the next it travels
//     through a per-group boundary row in global memory, read 32 columns ahead
//     by BoundaryPrefetch (hence the longer lag).
//
// A warp starts its next stripe when its previous one is done and the stripe
// above has been running long enough.  A stripe may end before the last
// column: the group keeps a column limit (the reverse region pass: the first
// begin-cell candidate; columns past it cannot change the result) that every
// running stripe applies at each chunk.  All warps read the limit a step
// published in the step before (two slots by step parity), so the stripes that
// run at the same time cut at the same column; a stripe is then never longer
// than the stripe above it, which keeps every producer at most 2 chunks ahead
// of its consumer.  Every group barrier is also a vote: the group leaves the
// loop when no warp has work.
#pragma once

#include "device_common.cuh"
#include "wavefront.cuh"

namespace ssa {

constexpr int PIPE_RING = 256;     // columns per boundary ring buffer (the producer runs 2 chunks ahead)

// Barrier of the W warps of group g (named barrier 1 + g of the CTA; a warp
// barrier when W == 1).  and_all(p): barrier that also returns p && ... over
// the group.
template <int W>
struct GroupBarrier {
    uint32_t id;
    __device__ void sync() const {
        if( W == 1 )
            __syncwarp();
        else
            asm volatile( "bar.sync %0, %1;" ::"r"( id ), "r"( W * 32 ) : "memory" );
    }
    __device__ bool and_all( bool p ) const {
        if( W == 1 )
            return __all_sync( 0xffffffffu, p );
        uint32_t r;
        asm volatile( "{\n\t.reg .pred pi, po;\n\t"
                      "setp.ne.u32 pi, %1, 0;\n\t"
                      "bar.red.and.pred po, %2, %3, pi;\n\t"
                      "selp.u32 %0, 1, 0, po;\n\t}"
                      : "=r"( r )
                      : "r"( (uint32_t) p ), "r"( id ), "r"( W * 32 )
                      : "memory" );
        return r != 0;
    }
};

// Shared state of one group.
template <int W>
struct PipeShared {
    int2 ring[W][2][PIPE_RING];    // bottom rows (H, F) of each warp's stripe, by super-pass parity
    int4 tiles[W][32];             // BoundaryPrefetch staging
    uint8_t residues[W][64];       // ResidueRing staging
    // per warp: the stripe it started most recently (low word, -1: none yet)
    // and the step it started at (high word), one 64-bit word so that a reader
    // never pairs a new stripe with an old step
    unsigned long long started[W];
    uint32_t item;                 // the group's current work item
    int32_t limit[2];              // column limit published for even / odd steps (INT32_MAX: none)
    int32_t red[W][4];             // per-warp results for the group reduction
};

// Where lane 0 of a stripe finds the row above it and where lane 31 puts the
// stripe's bottom row.
template <int W>
struct StripeLink {
    PipeShared<W> * sh;
    int4 * scratch;                // the group's global boundary row (scratch_cols entries)
    uint32_t scratch_cols;
    int wig;                       // warp in group
    uint32_t stripe;
    bool last;                     // no stripe below
    BoundaryPrefetch bp;
    // top row source: 0 = formula (stripe 0), 1 = global scratch, 2 = ring of warp wig - 1
    __device__ int source() const { return stripe == 0 ? 0 : (stripe % W == 0 ? 1 : 2); }
    __device__ void start( uint32_t cols, int lane ) {
        bp.tile = sh->tiles[wig];
        bp.start( scratch, scratch_cols, cols, source() == 1, lane );
    }
    __device__ void step( uint32_t cols, uint32_t s, int lane ) {
        bp.step( scratch, scratch_cols, cols, source() == 1, s, lane );
    }
    // (H, F) of the row above at column c (lane 0; source() != 0)
    __device__ int2 above( uint32_t s, int32_t c ) const {
        if( source() == 1 ) {
            const int4 v = bp.get( s );
            return make_int2( v.x, v.y );
        }
        const int pw = (wig + W - 1) % W;
        return sh->ring[pw][((stripe - 1) / W) & 1][c & (PIPE_RING - 1)];
    }
    // lane 31: the stripe's bottom row at column c; false if it did not fit
    __device__ bool put( int32_t c, int32_t h, int32_t f ) const {
        if( last )
            return true;
        if( stripe % W == W - 1 ) {
            if( (uint32_t) c >= scratch_cols )
                return false;
            scratch[c] = make_int4( h, f, 0, 0 );
        }
        else {
            sh->ring[wig][(stripe / W) & 1][c & (PIPE_RING - 1)] = make_int2( h, f );
        }
        return true;
    }
};

// Runs the stripes 0 .. n_stripes - 1 of one alignment on the group.  Body:
//   void begin( uint32_t stripe )          -- set up the warp's registers for a stripe
//   bool chunk( uint32_t c, int32_t lim )  -- wavefront steps 32c .. 32c + 31 (none
//                                             past column lim); false when the
//                                             stripe is done (after this chunk)
//   void end()                             -- fold the stripe's results into the warp's
//   int32_t cand                           -- the lane's limit candidate (INT32_MAX: none)
// Returns after the group barrier that ends the last step.  cols: database
// columns of the alignment; the schedule needs fewer than
// n_stripes x (chunks + 2W + 8) + 64 steps, and a loop that reaches that bound
// (which the schedule never does) sets ERR_PIPELINE and leaves, on every warp
// of the group at the same step.
template <int W, class Body>
__device__ void run_stripes( Body & body, PipeShared<W> & sh, const GroupBarrier<W> & gb, int wig, int lane,
        uint32_t n_stripes, uint32_t cols, unsigned * error_flags ) {
    const int64_t chunks = ((int64_t) cols + 31 + 31) / 32;
    const int64_t max_steps = (int64_t) n_stripes * (chunks + 2 * W + 8) + 64;
    if( lane == 0 )
        sh.started[wig] = 0xffffffffull;
    if( wig == 0 && lane == 0 ) {
        sh.limit[0] = INT32_MAX;
        sh.limit[1] = INT32_MAX;
    }
    gb.sync();
    uint32_t next = (uint32_t) wig;
    bool active = false;
    int32_t S = 0;
    for( int32_t T = 0;; T++ ) {
        if( !active && next < n_stripes ) {
            bool ok = (next == 0);
            if( !ok ) {
                const int pw = (wig + W - 1) % W;
                const int32_t lag = (next % W == 0) ? 4 : 2;
                const unsigned long long st = *(volatile unsigned long long *) &sh.started[pw];
                ok = (uint32_t) st == next - 1 && (int32_t) (st >> 32) <= T - lag;
            }
            if( ok ) {
                active = true;
                S = T;
                body.begin( next );
                __syncwarp();
                if( lane == 0 )
                    sh.started[wig] = ((unsigned long long) (uint32_t) T << 32) | next;
            }
        }
        const int32_t lim = sh.limit[T & 1];
        if( active ) {
            const bool more = body.chunk( (uint32_t) (T - S), lim );
            const int32_t m = __reduce_min_sync( 0xffffffffu, body.cand );
            if( lane == 0 && m < lim )
                atomicMin( &sh.limit[(T + 1) & 1], m );
            if( !more ) {
                body.end();
                active = false;
                next += W;
            }
        }
        if( wig == 0 && lane == 0 )
            atomicMin( &sh.limit[(T + 1) & 1], lim );
        if( gb.and_all( !active && next >= n_stripes ) )
            break;
        if( T >= max_steps ) {
            if( wig == 0 && lane == 0 )
                atomicOr( error_flags, ERR_PIPELINE );
            break;
        }
    }
}

}  // namespace ssa
