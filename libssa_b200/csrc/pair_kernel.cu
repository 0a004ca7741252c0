// pair_kernel.cu -- exact scores of long (query, database sequence) pairs.
//
// The inter-sequence passes give each database sequence to a few threads and
// need many sequences to fill the GPU; a batch of long pairs (a query against
// one chosen database sequence each, thousands of residues on both sides) has
// neither many sequences nor scores that fit 16 bits.  Here one warp aligns
// one pair as an anti-diagonal wavefront: lane k owns PAIR_R consecutive query
// rows of a stripe of 32 x PAIR_R rows, the database sequence streams through
// the warp (lane k works on column s - k at step s), a lane's bottom row
// reaches the next lane by shuffle, and a stripe's bottom row goes to a
// per-warp boundary row in global memory for the next stripe.
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
#include "wavefront.cuh"

namespace ssa {

constexpr int PAIR_ROWS = 32 * PAIR_R;
constexpr int PAIR_QS = 33;                       // score table row: 32 query codes + the past-the-end row
constexpr int32_t PAIR_PAST_END = -(1 << 20);     // score of rows past the query's end

// Score table [database code][query code] in shared memory, one row per
// database code.  The lanes of a warp read one row (the column's residue) at
// their own query codes, so distinct codes fall in distinct banks.  Column 32
// scores the rows past the query's end so low that they never hold a
// Smith-Waterman maximum (their values stay below the rows above them).
template <int ALGO>
__global__ void __launch_bounds__( PAIR_THREADS, 2 ) pair_score_kernel( PairScoreParams p ) {
    __shared__ int4 tiles[PAIR_THREADS / 32][32];
    __shared__ uint8_t rings[PAIR_THREADS / 32][64];
    __shared__ int32_t smat[32 * PAIR_QS];
    for( int i = threadIdx.x; i < 32 * PAIR_QS; i += blockDim.x ) {
        const int d = i / PAIR_QS, q = i % PAIR_QS;
        smat[i] = (q < 32) ? (int32_t) p.matrix[(d << 5) + q] : PAIR_PAST_END;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t w = blockIdx.x * (PAIR_THREADS / 32) + wib;
    int4 * scratch = p.scratch ? p.scratch + (uint64_t) w * p.scratch_cols : nullptr;
    const int32_t gO = p.gap_open, gE = p.gap_extend;
    const int32_t gOE = gO + gE;
    for( uint32_t t = next_hit( p.counter, lane ); t < p.n_pairs; t = next_hit( p.counter, lane ) ) {
        const uint32_t slot = p.pair_slot[t], unit = p.pair_unit[t];
        const uint32_t A = p.qlen[slot];
        const uint32_t B = p.db.lens[unit];
        const uint8_t * a = p.qcodes + p.qoff[slot];
        const uint8_t * b = p.db.codes + p.db.offsets[unit];
        const uint32_t stripes = (A + PAIR_ROWS - 1) / PAIR_ROWS;
        if( stripes > 1 && (scratch == nullptr || B > p.scratch_cols) ) {
            if( lane == 0 ) {
                atomicOr( p.error_flags, ERR_SCRATCH_OVERFLOW );
                p.score[t] = 0;
            }
            continue;
        }
        // Smith-Waterman: the maximum of the lane's cells; Needleman-Wunsch:
        // H(A - 1, B - 1) on the lane that owns row A - 1
        int32_t best = 0;
        for( uint32_t st = 0; st < stripes; st++ ) {
            const bool last = (st + 1 == stripes);
            const int32_t row0 = (int32_t) (st * PAIR_ROWS) + lane * PAIR_R;
            int qa[PAIR_R];
            int32_t H[PAIR_R], E[PAIR_R];
#pragma unroll
            for( int r = 0; r < PAIR_R; r++ ) {
                const int32_t i = row0 + r;
                qa[r] = (i < (int32_t) A) ? (int) a[i] : 32;
                // the reference's column before the first: H(i, -1), E(i, -1)
                H[r] = ALGO ? gO + (i + 1) * gE : 0;
                E[r] = ALGO ? 2 * gO + (i + 2) * gE : 0;
            }
            // H(row0 - 1, -1): the corner, or the boundary column above the lane
            int32_t diag = (ALGO && row0 > 0) ? gO + row0 * gE : 0;
            int32_t out_h = 0, out_f = 0;
            const int32_t rl = (int32_t) A - 1 - row0;   // Needleman-Wunsch: row A - 1 on this lane
            BoundaryPrefetch bp{ tiles[wib] };
            bp.start( scratch, p.scratch_cols, B, st > 0, lane );
            ResidueRing rr{ rings[wib], 0, b, (int32_t) B, -1 };
            rr.start( lane );
            for( uint32_t s = 0; s < B + 31; s++ ) {
                bp.step( scratch, p.scratch_cols, B, st > 0, s, lane );
                rr.step( s, lane );
                int32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
                int32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
                const int32_t c = (int32_t) s - lane;
                if( c < 0 || c >= (int32_t) B )
                    continue;
                if( lane == 0 ) {
                    if( st == 0 ) {
                        // the reference's row before the first: H(-1, c) (the
                        // next column's diagonal) and F(-1, c)
                        up_h = ALGO ? gO + (c + 1) * gE : 0;
                        up_f = ALGO ? 2 * gO + (c + 2) * gE : 0;
                    }
                    else {
                        const int4 v = bp.get( s );
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
                if( lane == 31 && !last )
                    scratch[c] = make_int4( out_h, out_f, 0, 0 );
                if( ALGO == 1 && last && c == (int32_t) B - 1 ) {
#pragma unroll
                    for( int r = 0; r < PAIR_R; r++ )
                        if( r == rl )
                            best = H[r];
                }
            }
            __syncwarp();
        }
        if( ALGO == 0 ) {
            best = __reduce_max_sync( 0xffffffffu, best );
        }
        else {
            const int owner = (int) (((A - 1u) % PAIR_ROWS) / PAIR_R);
            best = __shfl_sync( 0xffffffffu, best, owner );
        }
        if( lane == 0 )
            p.score[t] = best;
        __syncwarp();
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
