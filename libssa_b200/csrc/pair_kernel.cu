// pair_kernel.cu -- exact scores of long (query, database sequence) pairs.
//
// The inter-sequence passes give each database sequence to a few threads and
// need many sequences to fill the GPU; a batch of long pairs (a query against
// one chosen database sequence each, thousands of residues on both sides) has
// neither many sequences nor scores that fit 16 bits.  Here a group of PAIR_W
// warps aligns one pair as an anti-diagonal wavefront: lane k of a warp owns
// PAIR_R consecutive query rows of a stripe of 32 x PAIR_R rows, the database
// sequence streams through the warp (lane k works on column s - k at step s),
// a lane's bottom row reaches the next lane by shuffle, and consecutive
// stripes run on consecutive warps of the group, a stripe's bottom row handed
// to the next through shared memory or a per-group boundary row in global
// memory (stripe_pipeline.cuh).
//
// Values are int32, which the host guarantees to be exact for the pair's
// lengths and scores, so a pair gets the reference's 64-bit result
// (src/algo/64/smith_waterman_63.c:32-98, src/algo/64/needleman_wunsch_64.c:32-98):
// Smith-Waterman the maximum cell, Needleman-Wunsch the cell (qlen - 1,
// dlen - 1) under the reference's boundary rows and columns.  The entry widths
// of the reference report that same value for a database of one sequence (a
// saturated lane is re-searched at the next width), so this is what
// sw_align / nw_align return for the pair.
#include "device_common.cuh"
#include "stripe_pipeline.cuh"

namespace ssa {

constexpr int PAIR_ROWS = 32 * PAIR_R;
constexpr int PAIR_QS = 33;                       // score table row: 32 query codes + the past-the-end row
constexpr int32_t PAIR_PAST_END = -(1 << 20);     // score of rows past the query's end

// One stripe of a pair on one warp (the body run by run_stripes).  The score
// table [database code][query code] sits in shared memory, one row per
// database code: the lanes of a warp read one row (the column's residue) at
// their own query codes, so distinct codes fall in distinct banks.  Column 32
// scores the rows past the query's end so low that they never hold a
// Smith-Waterman maximum (their values stay below the rows above them).
template <int ALGO, int W>
struct PairStripe {
    const int32_t * smat;
    StripeLink<W> link;
    ResidueRing rr;
    const uint8_t * a;
    uint32_t A, B;
    int lane;
    int32_t gO, gE, gOE;
    unsigned * error_flags;
    int qa[PAIR_R];
    int32_t H[PAIR_R], E[PAIR_R];
    int32_t diag, out_h, out_f, row0;
    int32_t best;          // Smith-Waterman: the lane's maximum; Needleman-Wunsch: H(A - 1, B - 1) on its lane

    __device__ void begin( uint32_t stripe ) {
        link.stripe = stripe;
        link.last = (stripe + 1) * PAIR_ROWS >= A;
        row0 = (int32_t) (stripe * PAIR_ROWS) + lane * PAIR_R;
#pragma unroll
        for( int r = 0; r < PAIR_R; r++ ) {
            const int32_t i = row0 + r;
            qa[r] = (i < (int32_t) A) ? (int) a[i] : 32;
            // the reference's column before the first: H(i, -1), E(i, -1)
            H[r] = ALGO ? gO + (i + 1) * gE : 0;
            E[r] = ALGO ? 2 * gO + (i + 2) * gE : 0;
        }
        // H(row0 - 1, -1): the corner, or the boundary column above the lane
        diag = (ALGO && row0 > 0) ? gO + row0 * gE : 0;
        out_h = 0;
        out_f = 0;
        link.start( B, lane );
        rr.start( lane );
    }

    static constexpr int32_t cand = INT32_MAX;

    __device__ bool chunk( uint32_t ck, int32_t ) {
        const uint32_t steps = B + 31;
        const uint32_t s0 = ck * 32;
        const int32_t rl = (int32_t) A - 1 - row0;    // Needleman-Wunsch: row A - 1 on this lane
        // one wavefront step; edge: some lane may be on a column outside 0..B-1
        auto column = [&]( const uint32_t s, const bool edge ) {
            int32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
            int32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
            const int32_t c = (int32_t) s - lane;
            if( edge && (c < 0 || c >= (int32_t) B) )
                return;
            if( lane == 0 ) {
                if( link.stripe == 0 ) {
                    // the reference's row before the first: H(-1, c) (the next
                    // column's diagonal) and F(-1, c)
                    up_h = ALGO ? gO + (c + 1) * gE : 0;
                    up_f = ALGO ? 2 * gO + (c + 2) * gE : 0;
                }
                else {
                    const int2 v = link.above( s, c );
                    up_h = v.x;
                    up_f = v.y;
                }
            }
            const int32_t * mrow = smat + rr.get( s, lane ) * PAIR_QS;
            int32_t f = up_f, hd = diag;
            int32_t x_prev = 0;
#pragma unroll
            for( int r = 0; r < PAIR_R; r++ ) {
                const int32_t e = E[r];
                const int32_t x = ALGO ? __viaddmax_s32( hd, mrow[qa[r]], max( e, f ) )
                                       : __viaddmax_s32( hd, mrow[qa[r]], __vimax3_s32( e, f, 0 ) );
                hd = H[r];
                H[r] = x;
                const int32_t y = x + gOE;
                f = __viaddmax_s32( f, gE, y );
                E[r] = __viaddmax_s32( e, gE, y );
                if( ALGO == 0 ) {
                    if( r & 1 )
                        best = __vimax3_s32( best, x_prev, x );
                    else
                        x_prev = x;
                }
            }
            diag = up_h;
            out_h = H[PAIR_R - 1];
            out_f = f;
            if( lane == 31 && !link.put( c, out_h, out_f ) )
                atomicOr( error_flags, ERR_SCRATCH_OVERFLOW );
            if( ALGO == 1 && link.last && c == (int32_t) B - 1 ) {
#pragma unroll
                for( int r = 0; r < PAIR_R; r++ )
                    if( r == rl )
                        best = H[r];
            }
        };
        // the residue ring and the boundary prefetch refill at the first step of a chunk
        link.step( B, s0, lane );
        rr.step( s0, lane );
        const uint32_t s1 = min( s0 + 32, steps );
        if( s0 >= 31 && s1 <= B ) {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, false );
        }
        else {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, true );
        }
        return s0 + 32 < steps;
    }

    __device__ void end() {}
};

// A group of PAIR_W warps scores one pair at a time (stripe_pipeline.cuh).
template <int ALGO>
__global__ void __launch_bounds__( PAIR_THREADS, 2 ) pair_score_kernel( PairScoreParams p ) {
    constexpr int W = PAIR_W;
    constexpr int GROUPS = PAIR_THREADS / (32 * W);
    __shared__ PipeShared<W> shs[GROUPS];
    __shared__ int32_t smat[32 * PAIR_QS];
    for( int i = threadIdx.x; i < 32 * PAIR_QS; i += blockDim.x ) {
        const int d = i / PAIR_QS, q = i % PAIR_QS;
        smat[i] = (q < 32) ? (int32_t) p.matrix[(d << 5) + q] : PAIR_PAST_END;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = warp / W, wig = warp % W;
    PipeShared<W> & sh = shs[g];
    const GroupBarrier<W> gb{ 1u + (uint32_t) g };
    const uint64_t group = (uint64_t) blockIdx.x * GROUPS + g;
    int4 * scratch = p.scratch ? p.scratch + group * p.scratch_cols : nullptr;
    for( ;; ) {
        if( wig == 0 && lane == 0 )
            sh.item = (uint32_t) atomicAdd( p.counter, 1ull );
        gb.sync();
        const uint32_t t = sh.item;
        if( t >= p.n_pairs )
            break;
        const uint32_t slot = p.pair_slot[t], unit = p.pair_unit[t];
        PairStripe<ALGO, W> body;
        body.smat = smat;
        body.A = p.qlen[slot];
        body.B = p.db.lens[unit];
        body.a = p.qcodes + p.qoff[slot];
        body.lane = lane;
        body.gO = p.gap_open;
        body.gE = p.gap_extend;
        body.gOE = p.gap_open + p.gap_extend;
        body.error_flags = p.error_flags;
        body.best = 0;
        body.link.sh = &sh;
        body.link.scratch = scratch;
        body.link.scratch_cols = scratch ? p.scratch_cols : 0;
        body.link.wig = wig;
        body.rr = ResidueRing{ sh.residues[wig], 0, p.db.codes + p.db.offsets[unit], (int32_t) body.B, -1 };
        const uint32_t stripes = (body.A + PAIR_ROWS - 1) / PAIR_ROWS;
        run_stripes<W>( body, sh, gb, wig, lane, stripes, body.B, p.error_flags );
        // group result: the maximum over the warps, or the value of the lane
        // that owns cell (A - 1, B - 1)
        int32_t v = body.best;
        if( ALGO == 0 ) {
            v = __reduce_max_sync( 0xffffffffu, v );
            if( lane == 0 )
                sh.red[wig][0] = v;
        }
        else {
            const uint32_t owner_warp = (stripes - 1) % W;
            const int owner_lane = (int) (((body.A - 1u) % PAIR_ROWS) / PAIR_R);
            if( (uint32_t) wig == owner_warp && lane == owner_lane )
                sh.red[0][0] = v;
        }
        gb.sync();
        if( wig == 0 && lane == 0 ) {
            int32_t r = sh.red[0][0];
            if( ALGO == 0 )
                for( int k = 1; k < W; k++ )
                    r = max( r, sh.red[k][0] );
            p.score[t] = r;
        }
        // the next item is taken after every warp has read this one's results
        gb.sync();
    }
}

template <int ALGO>
static cudaError_t launch_pair_one( const PairScoreParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    if( blocks_per_sm )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, pair_score_kernel<ALGO>, PAIR_THREADS,
                0 );
    pair_score_kernel<ALGO><<<grid, PAIR_THREADS, 0, st>>>( p );
    return cudaGetLastError();
}

// blocks_per_sm != nullptr: only report the occupancy of the launch.
cudaError_t launch_pair_score( int algo, const PairScoreParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    return algo == 0 ? launch_pair_one<0>( p, grid, st, blocks_per_sm )
                     : launch_pair_one<1>( p, grid, st, blocks_per_sm );
}

}  // namespace ssa
