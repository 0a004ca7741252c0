// sw_fast_kernel.cu -- the Smith-Waterman 8-bit-entry search pass.
//
// The CPU library scores every database sequence first in a lane of a
// biased, saturating int8 vector kernel (reference:
// src/algo/simd/search_simd_sw.c:172-441): a lane reports score S if its
// running maximum never reached 255, and otherwise flags an overflow at the
// end of the first 4-column block in which it did; the sequence then goes to
// the 16-bit pass.  For Smith-Waterman that saturating arithmetic equals exact
// arithmetic with a floor at 0 as long as the running maximum stays below 255
// (the lower saturation is the SW zero floor, and an upward saturation can only
// happen in the cell that first reaches 255, which flags the overflow in the
// same block).  So this kernel computes exact 16-bit scores and records, per
// sequence, the first column where the running maximum reaches 255; its block
// index is the reference lane's overflow block.  This holds when the gap
// extension is <= 0 and the truncated 8-bit open+extend cost is in [-128, 0];
// the host routes other parameters to the exact lane emulation kernel.
//
// Mapping onto sm_100:
//   * two database sequences of similar length share each 32-bit register as
//     16x2 lanes (the database is packed once as length-sorted pairs with
//     interleaved residues);
//   * a group of G threads computes one pair as a wavefront: thread k holds
//     query rows [pass*G*R + k*R, +R) in registers and works on column
//     step-k; the bottom row's H and F and the running column maximum go to
//     thread k+1 by shuffle;
//   * the query profile (int8, 32 residue codes x padded rows) sits in shared
//     memory; per cell a PRMT sign-extends the two sequences' scores into a
//     16x2 word;
//   * all values carry a +1024 bias per half, so an add of gapO + gapE is a
//     plain 32-bit IADD (no borrow can cross halves: H never drops below the
//     bias) and the SW zero floor is a max with the bias;  per 16x2 cell
//     pair: one PRMT, three maxes, three fused add-max (all on the ALU pipe,
//     16 lanes per clock per SM sub-partition) and two IADDs (ALU or FMA
//     pipe), with a one-instruction dependency from row to row;
//   * every warp schedules itself: it takes (query, range of pairs) units from
//     a global counter, keeps the current pass's rows of the query profile in
//     its own shared-memory slice, and never waits on other warps;
//   * queries longer than G*R rows take several passes; the bottom row of a
//     pass goes through a per-group scratch row in global memory.
#include "device_common.cuh"

namespace ssa {

constexpr uint32_t FAST_BIAS = 1024u;
constexpr uint32_t FAST_BIAS2 = (FAST_BIAS << 16) | FAST_BIAS;
constexpr int FAST_THRESHOLD = 255;           // 8-bit lane overflow: running max reaches 255

__device__ __forceinline__ uint32_t prmt( uint32_t a, uint32_t b, uint32_t sel ) {
    uint32_t d;
    asm( "prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel) );
    return d;
}

// selector building (a.byte_j, sign(a.byte_j), b.byte_j, sign(b.byte_j))
__device__ __forceinline__ constexpr uint32_t sx_sel( int j ) {
    return (uint32_t) j | ((uint32_t) (j | 8) << 4) | ((uint32_t) (4 + j) << 8) | ((uint32_t) (12 + j) << 12);
}

template <int R>
struct ProfLoad {
    // loads R int8 profile entries starting at a 8-byte aligned shared address
    __device__ __forceinline__ static void load( const int8_t * p, uint32_t (&w)[R / 4] ) {
        if constexpr( R % 16 == 0 ) {
#pragma unroll
            for( int i = 0; i < R / 16; i++ ) {
                uint4 x = reinterpret_cast<const uint4 *>( p )[i];
                w[4 * i + 0] = x.x;
                w[4 * i + 1] = x.y;
                w[4 * i + 2] = x.z;
                w[4 * i + 3] = x.w;
            }
        }
        else {
#pragma unroll
            for( int i = 0; i < R / 8; i++ ) {
                uint2 x = reinterpret_cast<const uint2 *>( p )[i];
                w[2 * i + 0] = x.x;
                w[2 * i + 1] = x.y;
            }
        }
    }
};

template <int R>
__global__ void __launch_bounds__( 128, 4 ) sw_fast_kernel( FastParams p ) {
    // one profile slice (32 codes x G*R rows, G <= 32) per warp
    extern __shared__ __align__( 16 ) int8_t sprof[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int8_t * slice = sprof + (size_t) warp_in_cta * 32u * p.slice_rows;
    // per warp: the previous pass's boundary row, G columns per group, staged
    // ahead of use
    int4 * tiles = reinterpret_cast<int4 *>( sprof + (size_t) (FAST_THREADS / 32) * 32u * p.slice_rows ) +
            warp_in_cta * 32u;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) p.gap_e << 16) | (uint16_t) (int16_t) p.gap_e;
    const uint32_t TH = FAST_BIAS + FAST_THRESHOLD;
    uint64_t loaded_key = ~0ull;

    for( ;; ) {
        // a work unit: one query slot against one range of pairs
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t slot = p.unit_slots[u % p.n_class];
        const uint32_t chunk = (uint32_t) (u / p.n_class);
        const uint32_t pair_begin = p.chunk_bounds[chunk], pair_end = p.chunk_bounds[chunk + 1];
        const int G = (int) p.slot_group[slot];
        const uint32_t GR = (uint32_t) (G * R);
        const uint32_t rows = p.slot_rows[slot];
        const uint32_t passes = rows / GR;
        const int GPW = 32 / G;
        const int k = lane % G;                      // thread within its group
        const int g = lane / G;                      // group within the warp
        const int8_t * prof = p.prof8 + p.prof8_off[slot];
        int4 * scratch = p.scratch + ((uint64_t) warp_global * 4u + (uint32_t) g) * p.scratch_cols;

        for( uint32_t b0 = pair_begin; b0 < pair_end; b0 += (uint32_t) GPW ) {
            const uint32_t pair = b0 + (uint32_t) g;
            const bool valid = pair < pair_end;
            const uint32_t cols = valid ? p.pair_cols[pair] : 0u;
            const uint32_t max_cols = __reduce_max_sync( 0xffffffffu, cols );
            const uint8_t * res = p.pair_res + (valid ? p.pair_off[pair] : 0ull);

            int cross_lo = -1, cross_hi = -1;
            uint32_t final_s = FAST_BIAS2;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool final_pass = (pass + 1 == passes);
                // stage this pass's rows of the profile in the warp's slice
                const uint64_t key = ((uint64_t) slot << 16) | pass;
                if( key != loaded_key ) {
                    const uint32_t per_code = GR / 16u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < 32u * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 16u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                const uint32_t row_in_slice = (uint32_t) (k * R);
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = FAST_BIAS2;
                    E[r] = FAST_BIAS2;
                }
                uint32_t diag = FAST_BIAS2, smax = FAST_BIAS2;
                uint32_t out_h = FAST_BIAS2, out_f = FAST_BIAS2, out_s = FAST_BIAS2;
                // residues of columns c .. c+3 (two bytes each), refilled one
                // column ahead every step
                uint32_t q0 = 0, q1 = 0, q2 = 0, q3 = 0;
                {
                    const int32_t c0 = -k;
                    auto fetch = [&]( int32_t col ) -> uint32_t {
                        return (col >= 0 && (uint32_t) col < cols)
                                ? (uint32_t) *reinterpret_cast<const uint16_t *>( res + 2u * (uint32_t) col ) : 0u;
                    };
                    q0 = fetch( c0 );
                    q1 = fetch( c0 + 1 );
                    q2 = fetch( c0 + 2 );
                    q3 = fetch( c0 + 3 );
                }
                // boundary row of the previous pass: each lane of a group
                // prefetches one column, published to the group's tile every G steps
                int4 pf = make_int4( 0, 0, 0, 0 );
                int4 * tile = tiles + g * G;
                if( pass > 0 && (uint32_t) k < p.scratch_cols && (uint32_t) k < cols )
                    pf = scratch[k];
                const uint32_t steps = max_cols + (uint32_t) G - 1u;
                const uint32_t gmask = (uint32_t) G - 1u;    // G is a power of two
                for( uint32_t s = 0; s < steps; s++ ) {
                    if( pass > 0 && (s & gmask) == 0 ) {
                        __syncwarp();
                        tile[k] = pf;
                        __syncwarp();
                        const uint32_t col = s + (uint32_t) G + (uint32_t) k;
                        if( col < p.scratch_cols && col < cols )
                            pf = scratch[col];
                    }
                    uint32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1, G );
                    uint32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1, G );
                    uint32_t up_s = __shfl_up_sync( 0xffffffffu, out_s, 1, G );
                    const int32_t c = (int32_t) s - k;
                    const uint32_t w = q0;
                    q0 = q1;
                    q1 = q2;
                    q2 = q3;
                    {
                        // columns past the pair read its pad or the next pair's
                        // residues (never used); the buffer has 16 bytes of slack
                        const uint32_t col = min( (uint32_t) max( c + 4, 0 ), cols + 3u );
                        q3 = (uint32_t) *reinterpret_cast<const uint16_t *>( res + 2u * col );
                    }
                    if( c < 0 || (uint32_t) c >= cols )
                        continue;
                    if( k == 0 ) {
                        const int4 v = tile[s & gmask];
                        up_h = pass ? (uint32_t) v.x : FAST_BIAS2;
                        up_f = pass ? (uint32_t) v.y : FAST_BIAS2;
                        up_s = pass ? (uint32_t) v.z : FAST_BIAS2;
                    }
                    const uint32_t da = w & 0xffu;
                    const uint32_t db = w >> 8;
                    uint32_t pa[R / 4], pb[R / 4];
                    ProfLoad<R>::load( slice + da * GR + row_in_slice, pa );
                    ProfLoad<R>::load( slice + db * GR + row_in_slice, pb );
                    uint32_t f = up_f, hd = diag;
#pragma unroll
                    for( int r = 0; r < R; r++ ) {
                        // a = max(Hdiag + V, E, 0); since gapO <= 0 the next
                        // row's F only needs a: F' = max(F + gapE, a + gapO + gapE),
                        // so the row-to-row chain is one instruction
                        const uint32_t v = prmt( pa[r >> 2], pb[r >> 2], sx_sel( r & 3 ) );
                        const uint32_t e0 = __vmaxs2( E[r], FAST_BIAS2 );
                        const uint32_t a = __viaddmax_s16x2( hd, v, e0 );
                        const uint32_t h = __vmaxs2( a, f );                // H = max(a, F)
                        f = __viaddmax_s16x2( f, GE2, a + GOE32 );          // both halves, no borrow
                        E[r] = __viaddmax_s16x2( E[r], GE2, h + GOE32 );
                        hd = H[r];
                        H[r] = h;
                        smax = __vmaxs2( smax, h );
                    }
                    diag = up_h;
                    out_h = H[R - 1];
                    out_f = f;
                    out_s = __vmaxs2( up_s, smax );
                    if( k == G - 1 ) {
                        if( !final_pass ) {
                            if( (uint32_t) c < p.scratch_cols )
                                scratch[c] = make_int4( (int) out_h, (int) out_f, (int) out_s, 0 );
                            else
                                atomicOr( p.sink.error_flags, ERR_SCRATCH_OVERFLOW );
                        }
                        else {
                            if( cross_lo < 0 && (out_s & 0xffffu) >= TH )
                                cross_lo = c;
                            if( cross_hi < 0 && (out_s >> 16) >= TH )
                                cross_hi = c;
                            final_s = out_s;
                        }
                    }
                }
                __syncwarp();
            }
            // the group's last thread reports both sequences of the pair
            if( valid && k == G - 1 ) {
                const uint2 ids = p.pair_ids[pair];
                const uint32_t idv[2] = { ids.x, ids.y };
                const int cross[2] = { cross_lo, cross_hi };
                const uint32_t sv[2] = { final_s & 0xffffu, final_s >> 16 };
#pragma unroll
                for( int h = 0; h < 2; h++ ) {
                    if( idv[h] == 0xffffffffu )
                        continue;
                    if( cross[h] < 0 ) {
                        p.sink.score[(uint64_t) slot * p.sink.score_stride + idv[h]] = (int32_t) (sv[h] - FAST_BIAS);
                    }
                    else {
                        p.sink.score[(uint64_t) slot * p.sink.score_stride + idv[h]] = FAST_THRESHOLD;
                        unsigned q = atomicAdd( p.sink.next_count, 1u );
                        if( q < p.sink.next_cap )
                            p.sink.next[q] = PairTask{ slot, idv[h], cross[h] / 4 + 1, 0 };
                        else
                            atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                    }
                }
            }
        }
    }
}

// grid == 0: report the resident CTAs per SM in *blocks_per_sm without launching.
template <int R>
static cudaError_t launch_one( const FastParams & p, int grid, size_t smem, cudaStream_t st, int * blocks_per_sm ) {
    cudaError_t e = cudaFuncSetAttribute( sw_fast_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, sw_fast_kernel<R>, FAST_THREADS, smem );
    sw_fast_kernel<R><<<grid, FAST_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_sw_fast( int R, const FastParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    // one profile slice and one 32-entry boundary tile per warp
    const size_t smem = (size_t) (FAST_THREADS / 32) * (32u * p.slice_rows + 32u * sizeof(int4));
    switch( R ) {
    case 8:
        return launch_one<8>( p, grid, smem, st, blocks_per_sm );
    case 16:
        return launch_one<16>( p, grid, smem, st, blocks_per_sm );
    case 24:
        return launch_one<24>( p, grid, smem, st, blocks_per_sm );
    case 32:
        return launch_one<32>( p, grid, smem, st, blocks_per_sm );
    default:
        return cudaErrorInvalidValue;
    }
}

// ---- four columns per step ------------------------------------------------
// The same pass with one 4-column block per step: thread k of a group works
// on block step - k and interleaves the block's four columns row by row (cell
// (r, c + j) in row iteration r + j), so a thread carries four independent
// dependency chains and the recurrence can take its cheaper form
//     H = max(Hdiag + V, max(E, F, 0)),  E' / F' = max(E / F + gapE, H + gapO + gapE),
// two ALU instructions for H (3-way max, fused add-max), one IADD shared by
// both gap updates and two fused add-max: with the PRMT that builds the 16x2
// profile word and half a 3-way max for the running maximum, 5.5 ALU
// instructions and one IADD per cell pair (the one-column kernel above needs
// 7 and 2 to keep its row-to-row chain at one instruction).  Each thread
// records the first block in which its own running maximum reached 255; the
// group's minimum over threads and passes is the reference lane's overflow
// block.  A block's residues are one 8-byte load (4 columns x 2 sequences),
// read with the streaming cache operator; the boundary row of a multi-pass
// query (H and F of four columns, 32 bytes per block) goes through the
// group's scratch row, thread 0 reading it one block ahead.  G (threads per
// pair) is 4, 8, 16 or 32, so a warp holds up to 8 groups; R is 8, 16 or 24.
constexpr uint32_t FAST_CROSS_ADD =
        ((0x8000u - (FAST_BIAS + FAST_THRESHOLD)) << 16) | (0x8000u - (FAST_BIAS + FAST_THRESHOLD));

template <int R>
__global__ void __launch_bounds__( 128, 4 ) sw_fast4_kernel( FastParams p ) {
    constexpr int C = 4;
    extern __shared__ __align__( 16 ) int8_t sprof[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int8_t * slice = sprof + (size_t) warp_in_cta * 32u * p.slice_rows;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) p.gap_e << 16) | (uint16_t) (int16_t) p.gap_e;
    uint64_t loaded_key = ~0ull;

    for( ;; ) {
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t slot = p.unit_slots[u % p.n_class];
        const uint32_t chunk = (uint32_t) (u / p.n_class);
        const uint32_t pair_begin = p.chunk_bounds[chunk], pair_end = p.chunk_bounds[chunk + 1];
        const int G = (int) p.slot_group[slot];
        const uint32_t GR = (uint32_t) (G * R);
        const uint32_t rows = p.slot_rows[slot];
        const uint32_t passes = rows / GR;
        const int GPW = 32 / G;
        const int k = lane % G;
        const int g = lane / G;
        const int8_t * prof = p.prof8 + p.prof8_off[slot];
        int4 * scratch = p.scratch + ((uint64_t) warp_global * 8u + (uint32_t) g) * p.scratch_cols;

        for( uint32_t b0 = pair_begin; b0 < pair_end; b0 += (uint32_t) GPW ) {
            const uint32_t pair = b0 + (uint32_t) g;
            const bool valid = pair < pair_end;
            const uint32_t nb = valid ? p.pair_cols[pair] >> 2 : 0u;      // 4-column blocks
            const uint32_t max_nb = __reduce_max_sync( 0xffffffffu, nb );
            const uint8_t * res = p.pair_res + (valid ? p.pair_off[pair] : 0ull);

            uint32_t best = FAST_BIAS2;
            int cross_lo = INT_MAX, cross_hi = INT_MAX;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool last_pass = (pass + 1 == passes);
                const uint64_t key = ((uint64_t) slot << 16) | pass;
                if( key != loaded_key ) {
                    __syncwarp();
                    const uint32_t per_code = GR / 16u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < 32u * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 16u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = FAST_BIAS2;
                    E[r] = FAST_BIAS2;
                }
                uint32_t diag = FAST_BIAS2, smax = FAST_BIAS2, seen = 0;
                uint32_t out_h[C], out_f[C];
#pragma unroll
                for( int j = 0; j < C; j++ ) {
                    out_h[j] = FAST_BIAS2;
                    out_f[j] = FAST_BIAS2;
                }
                // residues of blocks b .. b + 3 (8 bytes each: a0 b0 a1 b1 a2
                // b2 a3 b3), one block fetched ahead every step; outside the
                // pair the reads are clamped to its blocks (never used)
                const uint32_t last_block = nb ? nb - 1u : 0u;
                auto fetch = [&]( int32_t b ) -> uint2 {
                    const uint32_t c = min( (uint32_t) max( b, 0 ), last_block );
                    return __ldcs( reinterpret_cast<const uint2 *>( res + 8u * c ) );
                };
                uint2 q0 = fetch( -k ), q1 = fetch( 1 - k ), q2 = fetch( 2 - k ), q3 = fetch( 3 - k );
                const bool reads_boundary = (k == 0) && pass > 0;
                int4 bq0 = make_int4( 0, 0, 0, 0 ), bq1 = bq0;
                if( reads_boundary && nb > 0 ) {
                    bq0 = scratch[0];
                    bq1 = scratch[1];
                }
                const uint32_t row0 = (uint32_t) (k * R);
                const uint32_t steps = max_nb + (uint32_t) G - 1u;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h[C], up_f[C];
#pragma unroll
                    for( int j = 0; j < C; j++ ) {
                        up_h[j] = __shfl_up_sync( 0xffffffffu, out_h[j], 1, G );
                        up_f[j] = __shfl_up_sync( 0xffffffffu, out_f[j], 1, G );
                    }
                    const int32_t b = (int32_t) s - k;
                    const uint2 w = q0;
                    q0 = q1;
                    q1 = q2;
                    q2 = q3;
                    q3 = fetch( b + 4 );
                    const int4 bnd0 = bq0, bnd1 = bq1;
                    if( reads_boundary ) {
                        const uint32_t nxt = (uint32_t) b + 1u;
                        if( nxt < nb && 2u * nxt + 1u < p.scratch_cols ) {
                            bq0 = scratch[2u * nxt];
                            bq1 = scratch[2u * nxt + 1u];
                        }
                    }
                    if( b < 0 || (uint32_t) b >= nb )
                        continue;
                    if( k == 0 ) {
                        if( pass ) {
                            up_h[0] = (uint32_t) bnd0.x;
                            up_f[0] = (uint32_t) bnd0.y;
                            up_h[1] = (uint32_t) bnd0.z;
                            up_f[1] = (uint32_t) bnd0.w;
                            up_h[2] = (uint32_t) bnd1.x;
                            up_f[2] = (uint32_t) bnd1.y;
                            up_h[3] = (uint32_t) bnd1.z;
                            up_f[3] = (uint32_t) bnd1.w;
                        }
                        else {
#pragma unroll
                            for( int j = 0; j < C; j++ ) {
                                up_h[j] = FAST_BIAS2;
                                up_f[j] = FAST_BIAS2;
                            }
                        }
                    }
                    // profile rows of column j's two residues
                    const int8_t * pa_base[C];
                    const int8_t * pb_base[C];
#pragma unroll
                    for( int j = 0; j < C; j++ ) {
                        const uint32_t word = j < 2 ? w.x : w.y;
                        const uint32_t sh = 16u * (uint32_t) (j & 1);
                        pa_base[j] = slice + ((word >> sh) & 0xffu) * GR + row0;
                        pb_base[j] = slice + ((word >> (sh + 8u)) & 0xffu) * GR + row0;
                    }
                    uint32_t pa[C], pb[C], f[C];
                    // hv[j][r]: H of chain j (column c + j) at row r; only the
                    // last two rows of chains 0..2 stay live
                    uint32_t hv[C][R];
#pragma unroll
                    for( int j = 0; j < C; j++ )
                        f[j] = up_f[j];
#pragma unroll
                    for( int it = 0; it < R + C - 1; it++ ) {
                        uint32_t hnew[C];
#pragma unroll
                        for( int j = 0; j < C; j++ ) {
                            const int r = it - j;
                            if( r < 0 || r >= R )
                                continue;
                            if( (r & 3) == 0 ) {
                                pa[j] = *reinterpret_cast<const uint32_t *>( pa_base[j] + r );
                                pb[j] = *reinterpret_cast<const uint32_t *>( pb_base[j] + r );
                            }
                            const uint32_t v = prmt( pa[j], pb[j], sx_sel( r & 3 ) );
                            uint32_t hd;
                            if( r == 0 )
                                hd = (j == 0) ? diag : up_h[j - 1];
                            else
                                hd = (j == 0) ? H[r - 1] : hv[j - 1][r - 1];
                            const uint32_t t = __vimax3_s16x2( E[r], f[j], FAST_BIAS2 );
                            const uint32_t h = __viaddmax_s16x2( hd, v, t );
                            const uint32_t hg = h + GOE32;                  // no borrow: h >= bias
                            f[j] = __viaddmax_s16x2( f[j], GE2, hg );
                            E[r] = __viaddmax_s16x2( E[r], GE2, hg );
                            hv[j][r] = h;
                            hnew[j] = h;
                        }
                        const int j0 = it - (R - 1) > 0 ? it - (R - 1) : 0;
                        const int j1 = it < C - 1 ? it : C - 1;
#pragma unroll
                        for( int j = j0; j <= j1; j += 2 ) {
                            if( j + 1 <= j1 )
                                smax = __vimax3_s16x2( smax, hnew[j], hnew[j + 1] );
                            else
                                smax = __vmaxs2( smax, hnew[j] );
                        }
                        // chain 3 leaves column c + 3 in H
                        if( it - (C - 1) >= 0 && it - (C - 1) < R )
                            H[it - (C - 1)] = hnew[C - 1];
                    }
                    diag = up_h[C - 1];
#pragma unroll
                    for( int j = 0; j < C; j++ ) {
                        out_h[j] = hv[j][R - 1];
                        out_f[j] = f[j];
                    }
                    // first block at which this thread's maximum reached 255
                    const uint32_t ge = (smax + FAST_CROSS_ADD) & 0x80008000u;
                    if( ge != seen ) {
                        if( (ge & 0x8000u) && !(seen & 0x8000u) )
                            cross_lo = min( cross_lo, b );
                        if( (ge & 0x80000000u) && !(seen & 0x80000000u) )
                            cross_hi = min( cross_hi, b );
                        seen = ge;
                    }
                    if( k == G - 1 && !last_pass ) {
                        if( 2u * (uint32_t) b + 1u < p.scratch_cols ) {
                            scratch[2u * b] = make_int4( (int) out_h[0], (int) out_f[0], (int) out_h[1],
                                    (int) out_f[1] );
                            scratch[2u * b + 1u] = make_int4( (int) out_h[2], (int) out_f[2], (int) out_h[3],
                                    (int) out_f[3] );
                        }
                        else {
                            atomicOr( p.sink.error_flags, ERR_SCRATCH_OVERFLOW );
                        }
                    }
                }
                best = __vmaxs2( best, smax );
                __syncwarp();
            }
            for( int o = 1; o < G; o <<= 1 ) {
                best = __vmaxs2( best, __shfl_xor_sync( 0xffffffffu, best, o, G ) );
                cross_lo = min( cross_lo, __shfl_xor_sync( 0xffffffffu, cross_lo, o, G ) );
                cross_hi = min( cross_hi, __shfl_xor_sync( 0xffffffffu, cross_hi, o, G ) );
            }
            if( valid && k == 0 ) {
                const uint2 ids = p.pair_ids[pair];
                const uint32_t idv[2] = { ids.x, ids.y };
                const int cross[2] = { cross_lo, cross_hi };
                const uint32_t sv[2] = { best & 0xffffu, best >> 16 };
#pragma unroll
                for( int h = 0; h < 2; h++ ) {
                    if( idv[h] == 0xffffffffu )
                        continue;
                    int32_t * dst = p.sink.score + (uint64_t) slot * p.sink.score_stride + idv[h];
                    if( cross[h] == INT_MAX ) {
                        *dst = (int32_t) (sv[h] - FAST_BIAS);
                    }
                    else {
                        *dst = FAST_THRESHOLD;
                        unsigned q = atomicAdd( p.sink.next_count, 1u );
                        if( q < p.sink.next_cap )
                            p.sink.next[q] = PairTask{ slot, idv[h], cross[h] + 1, 0 };
                        else
                            atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                    }
                }
            }
        }
    }
}

template <int R>
static cudaError_t launch_four( const FastParams & p, int grid, size_t smem, cudaStream_t st, int * blocks_per_sm ) {
    cudaError_t e = cudaFuncSetAttribute( sw_fast4_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, sw_fast4_kernel<R>, FAST_THREADS, smem );
    sw_fast4_kernel<R><<<grid, FAST_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_sw_fast4( int R, const FastParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    // one profile slice per warp
    const size_t smem = (size_t) (FAST_THREADS / 32) * 32u * p.slice_rows;
    switch( R ) {
    case 8:
        return launch_four<8>( p, grid, smem, st, blocks_per_sm );
    case 16:
        return launch_four<16>( p, grid, smem, st, blocks_per_sm );
    case 24:
        return launch_four<24>( p, grid, smem, st, blocks_per_sm );
    default:    // R = 32 would spill at 128 registers

        return cudaErrorInvalidValue;
    }
}

// prof8[slot][code][row]: the query's 8-bit scores, -128 past the query and for
// the neutral pad code used after a sequence's last 4-column block.
__global__ void build_profile8_kernel( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * slots, uint32_t n, const uint32_t * rows_of, const int64_t * matrix, int8_t * prof,
        const uint64_t * prof_off ) {
    const uint32_t i = blockIdx.y;
    if( i >= n )
        return;
    const uint32_t slot = slots[i];
    const uint32_t rows = rows_of[slot];
    const uint32_t Q = qlen[slot];
    const uint8_t * q = qcodes + qoff[slot];
    int8_t * out = prof + prof_off[slot];
    for( uint64_t x = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; x < 32ull * rows;
            x += (uint64_t) gridDim.x * blockDim.x ) {
        const uint32_t code = (uint32_t) (x / rows), row = (uint32_t) (x % rows);
        int8_t v = -128;
        if( row < Q && code != FAST_PAD_CODE )
            v = (int8_t) matrix[(code << 5) + q[row]];
        out[x] = v;
    }
}

cudaError_t launch_build_profile8( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * slots, uint32_t n, const uint32_t * rows_of, const int64_t * matrix, int8_t * prof,
        const uint64_t * prof_off, cudaStream_t st ) {
    if( n == 0 )
        return cudaSuccess;
    dim3 grid( 32, n );
    build_profile8_kernel<<<grid, 256, 0, st>>>( qcodes, qoff, qlen, slots, n, rows_of, matrix, prof, prof_off );
    return cudaGetLastError();
}

}  // namespace ssa
