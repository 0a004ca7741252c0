// traceback_kernels.cu -- CIGAR traceback of the top hits on the GPU.
//
// For every hit the CPU library runs three scalar O(q*d) passes and a walk
// (reference: src/algo/align.c:39-182, src/algo/cigar.c:48-346):
//
//   1. SW only: a forward local-alignment pass that finds the end cell, the
//      first cell (database-row major) holding the maximum;
//   2. SW only: a reverse pass from the end cell that finds the begin cell,
//      the first cell (scanning rows and columns downwards) whose value
//      reaches the score.  The reference resets its work rows only up to the
//      database end index, so when the query end lies beyond it the reverse
//      pass reads the forward pass's last-row values there; that is
//      reproduced exactly;
//   3. a direction pass over the matrix whose 4 flag bits collapse to the
//      three observable traceback moves, stored here as 2 bits per cell in HBM;
//   4. the walk from the end cell with the priority I > D > M.
//
// Each pass is a warp wavefront: lane k owns query rows [pass*256 + 8k, +8),
// database columns stream through the warp, the bottom row of a lane goes to
// the next lane by shuffle and the bottom row of a pass to a per-warp scratch
// row in global memory.  All arithmetic is exact (int32, with the host
// guaranteeing the range), matching the reference's int64 code.
#include "device_common.cuh"
#include "wavefront.cuh"

#include <climits>

namespace ssa {

constexpr int TB_R = TB_WORD_ROWS;   // query rows per lane (one direction word)
constexpr int TB_ROWS = 32 * TB_R;

// The 32x32 score table is staged in shared memory as int32 by every CTA,
// laid out [database code][query code] so that the lanes of a warp (different
// query rows, same database column) read different banks.  transposed = true
// stores matrix[query][db] there (the region passes score [query][db]).
__device__ __forceinline__ void stage_matrix( const int64_t * m, int32_t * sm, bool transposed ) {
    for( int i = threadIdx.x; i < 1024; i += blockDim.x ) {
        const int d = i >> 5, q = i & 31;
        sm[i] = (int32_t) (transposed ? m[(q << 5) + d] : m[(d << 5) + q]);
    }
    __syncthreads();
}

__device__ __forceinline__ int32_t mget( const int32_t * sm, int dcode, int qcode ) {
    return sm[(dcode << 5) + qcode];
}

// The lane's R query codes (code 0 past the end) held in registers.
__device__ __forceinline__ void load_rows( const uint8_t * a, int64_t first, int64_t step, int nvalid,
        int (&code)[TB_R] ) {
#pragma unroll
    for( int r = 0; r < TB_R; r++ )
        code[r] = (r < nvalid) ? a[first + step * r] : 0;
}


// ---------------------------------------------------------------------------
// 1. SW forward region pass (reference: src/algo/align.c:39-82).  The
//    reference iterates database rows outer and query columns inner, scoring
//    matrix[query][db]; the recurrence is symmetric, so the warp streams the
//    database and keeps the query on lanes.  Key of the end cell: largest
//    value, then smallest database index, then smallest query index.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__( 256 ) tb_forward_kernel( TbParams p ) {
    __shared__ int4 tiles[8][32];
    __shared__ uint8_t rings[8][64];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, true );
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int4 * scratch = p.scratch + (uint64_t) w * p.scratch_cols;
    const int gO = p.gap_open, gE = p.gap_extend;
    const int gOE = gO + gE;
    for( uint32_t h = next_hit( p.hit_counters + 0, lane ); h < p.n_hits; h = next_hit( p.hit_counters + 0, lane ) ) {
        const TbHit hit = p.hits[h];
        if( hit.algo != 0 )
            continue;
        const uint32_t A = p.qlen[hit.qslot];
        const uint32_t B = p.db.lens[hit.id];
        const uint8_t * a = p.qcodes + p.qoff[hit.qslot];
        const uint8_t * b = p.db.codes + p.db.offsets[hit.id];
        int32_t * lh = p.last_h + p.last_off[h];
        int32_t * le = p.last_e + p.last_off[h];
        const uint32_t passes = (A + TB_ROWS - 1) / TB_ROWS;
        // best cell of this lane: value, db index, query index
        int32_t best_v = 0;
        int32_t best_i = INT_MAX, best_j = INT_MAX;
        for( uint32_t pass = 0; pass < passes; pass++ ) {
            const bool final_pass = (pass + 1 == passes);
            const int32_t row0 = (int32_t) (pass * TB_ROWS + lane * TB_R);
            const int nvalid = max( 0, min( TB_R, (int) A - row0 ) );
            int qa[TB_R];
            load_rows( a, row0, 1, nvalid, qa );
            int32_t H[TB_R], E[TB_R];
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                H[r] = 0;          // HH[j] = 0
                E[r] = gO + gE;    // max(EE = gapO, HH + gapO) + gapE at row 0
            }
            int32_t diag = 0;
            int32_t out_h = 0, out_f = 0;
            int32_t pv = 0, pi = INT_MAX, pj = INT_MAX;     // this pass's first maximum
            BoundaryPrefetch bp{ tiles[threadIdx.x >> 5] };
            bp.start( scratch, p.scratch_cols, B, pass > 0, lane );
            ResidueRing rr{ rings[threadIdx.x >> 5], 0, b, (int32_t) B, -1 };
            rr.start( lane );
            for( uint32_t s = 0; s < B + 31; s++ ) {
                bp.step( scratch, p.scratch_cols, B, pass > 0, s, lane );
                rr.step( s, lane );
                int32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
                int32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
                const int32_t c = (int32_t) s - lane;
                if( c < 0 || c >= (int32_t) B )
                    continue;
                if( lane == 0 ) {
                    if( pass == 0 ) {
                        up_h = 0;
                        up_f = gO + gE;   // f starts at gapO: max(gapO, 0 + gapO) + gapE
                    }
                    else {
                        const int4 v = bp.get( s );
                        up_h = v.x;
                        up_f = v.y;
                    }
                }
                int32_t f = up_f, hd = diag;
                const int d = rr.get( s, lane );
                // branch-free rows: the row-to-row chain is a 3-way max, an
                // add and a fused add-max; a lane visits its cells in (column,
                // row) order, so within a pass the first maximum wins with a
                // strict compare
                int32_t e_last[TB_R];
#pragma unroll
                for( int r = 0; r < TB_R; r++ ) {
                    const int32_t e_in = E[r];
                    const int32_t t = max( hd + mget( smat, d, qa[r] ), 0 );
                    const int32_t x = __vimax3_s32( t, f, e_in );
                    const bool take = (r < nvalid) && x > pv;
                    pv = take ? x : pv;
                    pi = take ? c : pi;
                    pj = take ? row0 + r : pj;
                    e_last[r] = e_in;
                    hd = H[r];
                    H[r] = x;
                    const int32_t y = x + gOE;
                    f = __viaddmax_s32( f, gE, y );
                    E[r] = __viaddmax_s32( e_in, gE, y );
                }
                if( c == (int32_t) B - 1 ) {
#pragma unroll
                    for( int r = 0; r < TB_R; r++ )
                        if( r < nvalid ) {
                            lh[row0 + r] = H[r];
                            le[row0 + r] = e_last[r];
                        }
                }
                diag = up_h;
                out_h = H[TB_R - 1];
                out_f = f;
                if( lane == 31 && !final_pass ) {
                    if( (uint32_t) c < p.scratch_cols )
                        scratch[c] = make_int4( out_h, out_f, 0, 0 );
                    else
                        atomicOr( p.error_flags, ERR_SCRATCH_OVERFLOW );
                }
            }
            // this pass's first maximum against the earlier passes' (value desc,
            // database index asc, query index asc)
            if( pv > best_v || (pv == best_v && pv > 0 && (pi < best_i || (pi == best_i && pj < best_j))) ) {
                best_v = pv;
                best_i = pi;
                best_j = pj;
            }
            __syncwarp();
        }
        // reduce the best key over the warp
        for( int o = 16; o > 0; o >>= 1 ) {
            int32_t v = __shfl_xor_sync( 0xffffffffu, best_v, o );
            int32_t bi = __shfl_xor_sync( 0xffffffffu, best_i, o );
            int32_t bj = __shfl_xor_sync( 0xffffffffu, best_j, o );
            if( v > best_v || (v == best_v && (bi < best_i || (bi == best_i && bj < best_j))) ) {
                best_v = v;
                best_i = bi;
                best_j = bj;
            }
        }
        if( lane == 0 ) {
            TbRegion rg;
            rg.fwd_score = best_v;
            rg.a_end = best_j;
            rg.b_end = best_i;
            rg.a_begin = 0;
            rg.b_begin = 0;
            rg.status = (best_v > 0) ? 0 : 1;
            p.regions[h] = rg;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 2. SW reverse pass (reference: src/algo/align.c:84-131).  Both sequences
//    are read backwards from the end cell: row j' = a_end - j, column
//    i' = b_end - i.  The boundary row before column 0 is the reference's
//    work row: -1 for query indices <= b_end, the forward pass's last row
//    above that.  The begin cell is the first cell in (i' asc, j' asc) order
//    whose value reaches the forward score.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__( 256 ) tb_reverse_kernel( TbParams p ) {
    __shared__ int4 tiles[8][32];
    __shared__ uint8_t rings[8][64];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, true );
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int4 * scratch = p.scratch + (uint64_t) w * p.scratch_cols;
    const int gO = p.gap_open, gE = p.gap_extend;
    const int gOE = gO + gE;
    for( uint32_t h = next_hit( p.hit_counters + 1, lane ); h < p.n_hits; h = next_hit( p.hit_counters + 1, lane ) ) {
        const TbHit hit = p.hits[h];
        if( hit.algo != 0 )
            continue;
        TbRegion rg = p.regions[h];
        if( rg.status != 0 )
            continue;
        const int32_t score = rg.fwd_score;
        const int32_t a_end = rg.a_end, b_end = rg.b_end;
        const uint32_t A = (uint32_t) a_end + 1;     // rows j' = 0..a_end
        const uint32_t B = (uint32_t) b_end + 1;     // cols i' = 0..b_end
        const uint8_t * a = p.qcodes + p.qoff[hit.qslot];
        const uint8_t * b = p.db.codes + p.db.offsets[hit.id];
        const int32_t * lh = p.last_h + p.last_off[h];
        const int32_t * le = p.last_e + p.last_off[h];
        const uint32_t passes = (A + TB_ROWS - 1) / TB_ROWS;
        int32_t hit_i = INT_MAX, hit_j = INT_MAX;   // first (i', j') reaching the score
        for( uint32_t pass = 0; pass < passes; pass++ ) {
            const bool final_pass = (pass + 1 == passes);
            const int32_t row0 = (int32_t) (pass * TB_ROWS + lane * TB_R);
            const int nvalid = max( 0, min( TB_R, (int) A - row0 ) );
            int qa[TB_R];
            load_rows( a, (int64_t) a_end - row0, -1, nvalid, qa );
            int32_t H[TB_R], E[TB_R];
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t j = a_end - (row0 + r);     // query index
                int32_t hh = -1, ee = -1;
                if( r < nvalid && j > b_end ) {
                    hh = lh[j];
                    ee = le[j];
                }
                H[r] = hh;                                // HH(b_end + 1, j)
                E[r] = max( ee, hh + gO ) + gE;           // EE(b_end, j)
            }
            // diagonal of the lane's first row at column 0: HH(b_end+1, j+1),
            // or 0 for the end cell itself
            int32_t diag;
            {
                const int32_t jprev = a_end - (row0 - 1);
                if( row0 == 0 )
                    diag = 0;
                else
                    diag = (jprev > b_end) ? lh[jprev] : -1;
            }
            int32_t out_h = 0, out_f = 0;
            // columns past the first one holding a begin-cell candidate cannot
            // change the result: stop once every lane has passed it
            int32_t limit = __reduce_min_sync( 0xffffffffu, hit_i );
            BoundaryPrefetch bp{ tiles[threadIdx.x >> 5] };
            bp.start( scratch, p.scratch_cols, B, pass > 0, lane );
            ResidueRing rr{ rings[threadIdx.x >> 5], 0, b, (int32_t) B, b_end };
            rr.start( lane );
            for( uint32_t s = 0; s < B + 31; s++ ) {
                if( (s & 7) == 0 )
                    limit = __reduce_min_sync( 0xffffffffu, hit_i );
                if( limit != INT_MAX && (int64_t) s > (int64_t) limit + 31 )
                    break;
                bp.step( scratch, p.scratch_cols, B, pass > 0, s, lane );
                rr.step( s, lane );
                int32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
                int32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
                const int32_t c = (int32_t) s - lane;
                if( c < 0 || c >= (int32_t) B )
                    continue;
                if( lane == 0 ) {
                    if( pass == 0 ) {
                        up_h = -1;                        // h starts at -1 per row
                        up_f = max( -1, -1 + gO ) + gE;   // f = max(-1, h + gapO) + gapE
                    }
                    else {
                        const int4 v = bp.get( s );
                        up_h = v.x;
                        up_f = v.y;
                    }
                }
                const int d = rr.get( s, lane );          // database index b_end - c
                int32_t f = up_f, hd = diag;              // lane 0 / pass 0: 0 at c == 0, then -1
#pragma unroll
                for( int r = 0; r < TB_R; r++ ) {
                    const int32_t e_in = E[r];
                    const int32_t x = __vimax3_s32( hd + mget( smat, d, qa[r] ), f, e_in );
                    const bool take = (r < nvalid) && x >= score &&
                            (c < hit_i || (c == hit_i && row0 + r < hit_j));
                    hit_i = take ? c : hit_i;
                    hit_j = take ? row0 + r : hit_j;
                    hd = H[r];
                    H[r] = x;
                    const int32_t y = x + gOE;
                    f = __viaddmax_s32( f, gE, y );
                    E[r] = __viaddmax_s32( e_in, gE, y );
                }
                diag = up_h;
                out_h = H[TB_R - 1];
                out_f = f;
                if( lane == 31 && !final_pass ) {
                    if( (uint32_t) c < p.scratch_cols )
                        scratch[c] = make_int4( out_h, out_f, 0, 0 );
                    else
                        atomicOr( p.error_flags, ERR_SCRATCH_OVERFLOW );
                }
            }
            __syncwarp();
        }
        for( int o = 16; o > 0; o >>= 1 ) {
            int32_t bi = __shfl_xor_sync( 0xffffffffu, hit_i, o );
            int32_t bj = __shfl_xor_sync( 0xffffffffu, hit_j, o );
            if( bi < hit_i || (bi == hit_i && bj < hit_j) ) {
                hit_i = bi;
                hit_j = bj;
            }
        }
        if( lane == 0 ) {
            if( hit_i == INT_MAX ) {
                rg.status = 2;
            }
            else {
                rg.b_begin = b_end - hit_i;
                rg.a_begin = a_end - hit_j;
            }
            p.regions[h] = rg;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 3. Direction pass (reference: src/algo/cigar.c:48-198).  Query rows on
//    lanes, database columns streamed, exactly the reference orientation.
//    Codes: 0 = M, 1 = D (UP|EXT_UP), 2 = I (LEFT|EXT_LEFT, takes priority).
//    Stored for columns [b_begin, b_end] and all query rows of the lane, one
//    16-bit word (8 rows x 2 bits) per lane and column.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__( 256 ) tb_directions_kernel( TbParams p ) {
    __shared__ int4 tiles[8][32];
    __shared__ uint8_t rings[8][64];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, false );
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int4 * scratch = p.scratch + (uint64_t) w * p.scratch_cols;
    const int gO = p.gap_open, gE = p.gap_extend;
    const int gOE = gO + gE;
    for( uint32_t h = next_hit( p.hit_counters + 2, lane ); h < p.n_hits; h = next_hit( p.hit_counters + 2, lane ) ) {
        const TbHit hit = p.hits[h];
        const TbRegion rg = p.regions[h];
        if( rg.status != 0 )
            continue;
        const bool nw = hit.algo == 1;
        const uint32_t A = (uint32_t) rg.a_end + 1;   // rows 0..a_end suffice
        const uint32_t B = (uint32_t) rg.b_end + 1;   // columns 0..b_end
        const uint32_t words = (A + TB_R - 1) / TB_R;
        const uint8_t * a = p.qcodes + p.qoff[hit.qslot];
        const uint8_t * b = p.db.codes + p.db.offsets[hit.id];
        uint16_t * dir = p.dirs + p.dir_off[h];
        const uint32_t passes = (A + TB_ROWS - 1) / TB_ROWS;
        for( uint32_t pass = 0; pass < passes; pass++ ) {
            const bool final_pass = (pass + 1 == passes);
            const int32_t row0 = (int32_t) (pass * TB_ROWS + lane * TB_R);
            const int nvalid = max( 0, min( TB_R, (int) A - row0 ) );
            int qa[TB_R];
            load_rows( a, row0, 1, nvalid, qa );
            int32_t H[TB_R], E[TB_R];
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t i = row0 + r;
                H[r] = nw ? gO + (i + 1) * gE : 0;
                E[r] = nw ? 2 * gO + (i + 2) * gE : 0;
            }
            int32_t diag = nw ? ((row0 == 0) ? 0 : gO + row0 * gE) : 0;
            int32_t out_h = 0, out_f = 0;
            BoundaryPrefetch bp{ tiles[threadIdx.x >> 5] };
            bp.start( scratch, p.scratch_cols, B, pass > 0, lane );
            ResidueRing rr{ rings[threadIdx.x >> 5], 0, b, (int32_t) B, -1 };
            rr.start( lane );
            for( uint32_t s = 0; s < B + 31; s++ ) {
                bp.step( scratch, p.scratch_cols, B, pass > 0, s, lane );
                rr.step( s, lane );
                int32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
                int32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
                const int32_t j = (int32_t) s - lane;     // database index
                if( j < 0 || j >= (int32_t) B )
                    continue;
                if( lane == 0 ) {
                    if( pass == 0 ) {
                        // H(-1, j) is the next column's row-0 diagonal
                        up_h = nw ? gO + (j + 1) * gE : 0;
                        up_f = nw ? 2 * gO + (j + 2) * gE : 0;
                    }
                    else {
                        const int4 v = bp.get( s );
                        up_h = v.x;
                        up_f = v.y;
                    }
                }
                const int d = rr.get( s, lane );
                int32_t f = up_f, hd = diag;
                uint32_t code = 0;
                // flags as in the reference (strict compares in its order),
                // computed beside a branch-free row-to-row chain
#pragma unroll
                for( int r = 0; r < TB_R; r++ ) {
                    const int32_t e = E[r];
                    const int32_t x0 = hd + mget( smat, d, qa[r] );
                    const bool up = f > x0;                      // UP
                    const bool left = e > max( x0, f );          // LEFT
                    const int32_t x = __vimax3_s32( nw ? x0 : max( x0, 0 ), f, e );
                    hd = H[r];
                    H[r] = x;
                    const int32_t y = x + gOE;
                    const bool ext_up = f + gE > y;              // EXT_UP
                    const bool ext_left = e + gE > y;            // EXT_LEFT
                    f = __viaddmax_s32( f, gE, y );
                    E[r] = __viaddmax_s32( e, gE, y );
                    const uint32_t op = (left || ext_left) ? 2u : ((up || ext_up) ? 1u : 0u);
                    code |= (r < nvalid) ? op << (2 * r) : 0u;
                }
                diag = up_h;
                out_h = H[TB_R - 1];
                out_f = f;
                if( j >= rg.b_begin && (uint32_t) (row0 / TB_R) < words )
                    dir[(uint64_t) (j - rg.b_begin) * words + row0 / TB_R] = (uint16_t) code;
                if( lane == 31 && !final_pass ) {
                    if( (uint32_t) j < p.scratch_cols )
                        scratch[j] = make_int4( out_h, out_f, 0, 0 );
                    else
                        atomicOr( p.error_flags, ERR_SCRATCH_OVERFLOW );
                }
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// 4. Walk (reference: src/algo/cigar.c:300-334): one thread per hit writes the
//    moves in traceback order (end to begin); the host run-length encodes.
// ---------------------------------------------------------------------------
__global__ void tb_walk_kernel( TbParams p ) {
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if( h >= p.n_hits )
        return;
    const TbRegion rg = p.regions[h];
    if( rg.status != 0 ) {
        p.ops_len[h] = 0;
        return;
    }
    const uint32_t words = ((uint32_t) rg.a_end + 1 + TB_R - 1) / TB_R;
    const uint16_t * dir = p.dirs + p.dir_off[h];
    char * out = p.ops + p.ops_off[h];
    const uint64_t cap = p.ops_off[h + 1] - p.ops_off[h];
    int64_t i = rg.a_end, j = rg.b_end;
    uint64_t n = 0;
    while( i >= rg.a_begin && j >= rg.b_begin && i >= 0 && j >= 0 ) {
        const uint32_t word = dir[(uint64_t) (j - rg.b_begin) * words + (uint64_t) (i / TB_R)];
        const uint32_t op = (word >> (2 * (i % TB_R))) & 3u;
        char ch;
        if( op == 2u ) {
            j--;
            ch = 'I';
        }
        else if( op == 1u ) {
            i--;
            ch = 'D';
        }
        else {
            i--;
            j--;
            ch = 'M';
        }
        if( n < cap )
            out[n] = ch;
        n++;
    }
    p.ops_len[h] = (uint32_t) n;
}

// Region phase (Smith-Waterman hits only): forward and reverse passes.  They
// need no direction memory, so all hits of a search run in one launch each.
// ev (optional): 3 events recorded around the two kernels.
cudaError_t launch_tb_regions( const TbParams & p, int grid, cudaStream_t st, cudaEvent_t * ev ) {
    if( ev )
        cudaEventRecord( ev[0], st );
    if( p.n_hits ) {
        tb_forward_kernel<<<grid, 256, 0, st>>>( p );
        if( ev )
            cudaEventRecord( ev[1], st );
        tb_reverse_kernel<<<grid, 256, 0, st>>>( p );
    }
    else if( ev ) {
        cudaEventRecord( ev[1], st );
    }
    if( ev )
        cudaEventRecord( ev[2], st );
    return cudaGetLastError();
}

// Path phase: direction pass and walk of the hits of one wave (the hits whose
// direction words fit the memory the host set aside).
// ev (optional): 3 events recorded around the two kernels.
cudaError_t launch_tb_paths( const TbParams & p, int grid, cudaStream_t st, cudaEvent_t * ev ) {
    if( ev )
        cudaEventRecord( ev[0], st );
    if( p.n_hits ) {
        tb_directions_kernel<<<grid, 256, 0, st>>>( p );
        if( ev )
            cudaEventRecord( ev[1], st );
        tb_walk_kernel<<<(p.n_hits + 127) / 128, 128, 0, st>>>( p );
    }
    else if( ev ) {
        cudaEventRecord( ev[1], st );
    }
    if( ev )
        cudaEventRecord( ev[2], st );
    return cudaGetLastError();
}

}  // namespace ssa
