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
//   * all values carry a +1024 bias per half, so H + gapO + gapE is a plain
//     32-bit IADD (no borrow can cross halves) and the SW zero floor is a
//     max with the bias;  per 16x2 cell pair: 4 half-rate DPX/PRMT and
//     4 full-rate instructions;
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

template <int R, int G>
__global__ void __launch_bounds__( 256, 1 ) sw_fast_kernel( FastParams p ) {
    extern __shared__ __align__( 16 ) int8_t sprof[];
    __shared__ FastItem cur;
    __shared__ unsigned pair_next;
    __shared__ uint32_t loaded_slot;

    constexpr int GPW = 32 / G;                  // groups per warp
    const int lane = threadIdx.x & 31;
    const int k = lane % G;                      // thread within its group
    const int g = lane / G;                      // group within the warp
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t rows = p.rows;
    const uint32_t passes = p.passes;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) p.gap_e << 16) | (uint16_t) (int16_t) p.gap_e;
    const uint32_t TH = FAST_BIAS + FAST_THRESHOLD;
    int4 * scratch = p.scratch + ((uint64_t) warp_global * GPW + g) * p.scratch_cols;

    if( threadIdx.x == 0 )
        loaded_slot = 0xffffffffu;
    for( ;; ) {
        __syncthreads();
        if( threadIdx.x == 0 ) {
            unsigned it = atomicAdd( p.item_counter, 1u );
            if( it < p.n_items ) {
                cur = p.items[it];
            }
            else {
                cur.slot = 0xffffffffu;
                cur.pair_begin = cur.pair_end = 0;
            }
            pair_next = cur.pair_begin;
        }
        __syncthreads();
        if( cur.slot == 0xffffffffu )
            break;
        if( cur.slot != loaded_slot ) {
            const uint4 * src = reinterpret_cast<const uint4 *>( p.prof8 + p.prof8_off[cur.slot] );
            uint4 * dst = reinterpret_cast<uint4 *>( sprof );
            const uint32_t n16 = 32u * rows / 16u;
            for( uint32_t i = threadIdx.x; i < n16; i += blockDim.x )
                dst[i] = src[i];
            __syncthreads();
            if( threadIdx.x == 0 )
                loaded_slot = cur.slot;
        }
        const uint32_t slot = cur.slot;

        for( ;; ) {
            unsigned b0 = 0;
            if( lane == 0 )
                b0 = atomicAdd( &pair_next, (unsigned) GPW );
            b0 = __shfl_sync( 0xffffffffu, b0, 0 );
            if( b0 >= cur.pair_end )
                break;
            const uint32_t pair = b0 + g;
            const bool valid = pair < cur.pair_end;
            const uint32_t cols = valid ? p.pair_cols[pair] : 0u;
            const uint32_t max_cols = __reduce_max_sync( 0xffffffffu, cols );
            const uint8_t * res = p.pair_res + (valid ? p.pair_off[pair] : 0ull);

            int cross_lo = -1, cross_hi = -1;
            uint32_t final_s = FAST_BIAS2;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool final_pass = (pass + 1 == passes);
                const uint32_t row0 = pass * (uint32_t) (G * R) + (uint32_t) (k * R);
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = FAST_BIAS2;
                    E[r] = FAST_BIAS2;
                }
                uint32_t diag = FAST_BIAS2, smax = FAST_BIAS2;
                uint32_t out_h = FAST_BIAS2, out_f = FAST_BIAS2, out_s = FAST_BIAS2;
                uint32_t rw = 0;
                const uint32_t steps = max_cols + G - 1;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h = __shfl_up_sync( 0xffffffffu, out_h, 1, G );
                    uint32_t up_f = __shfl_up_sync( 0xffffffffu, out_f, 1, G );
                    uint32_t up_s = __shfl_up_sync( 0xffffffffu, out_s, 1, G );
                    const int32_t c = (int32_t) s - k;
                    if( c < 0 || (uint32_t) c >= cols )
                        continue;
                    if( k == 0 ) {
                        if( pass == 0 ) {
                            up_h = FAST_BIAS2;
                            up_f = FAST_BIAS2;
                            up_s = FAST_BIAS2;
                        }
                        else {
                            int4 v = scratch[c];
                            up_h = (uint32_t) v.x;
                            up_f = (uint32_t) v.y;
                            up_s = (uint32_t) v.z;
                        }
                    }
                    if( (c & 1) == 0 )
                        rw = *reinterpret_cast<const uint32_t *>( res + 2 * (uint32_t) c );
                    const uint32_t sh = (uint32_t) (c & 1) * 16u;
                    const uint32_t da = (rw >> sh) & 0xffu;
                    const uint32_t db = (rw >> (sh + 8u)) & 0xffu;
                    uint32_t pa[R / 4], pb[R / 4];
                    ProfLoad<R>::load( sprof + da * rows + row0, pa );
                    ProfLoad<R>::load( sprof + db * rows + row0, pb );
                    uint32_t f = up_f, hd = diag;
#pragma unroll
                    for( int r = 0; r < R; r++ ) {
                        const uint32_t v = prmt( pa[r >> 2], pb[r >> 2], sx_sel( r & 3 ) );
                        uint32_t t = __vmaxs2( E[r], f );
                        t = __vmaxs2( t, FAST_BIAS2 );                    // SW floor at 0
                        const uint32_t h = __viaddmax_s16x2( hd, v, t );   // max(Hdiag + V, E, F, 0)
                        hd = H[r];
                        H[r] = h;
                        const uint32_t hg = h + GOE32;                     // H + gapO + gapE, both halves
                        E[r] = __viaddmax_s16x2( E[r], GE2, hg );
                        f = __viaddmax_s16x2( f, GE2, hg );
                        smax = __vmaxs2( smax, h );
                    }
                    diag = up_h;
                    out_h = H[R - 1];
                    out_f = f;
                    out_s = __vmaxs2( up_s, smax );
                    if( k == G - 1 ) {
                        if( !final_pass ) {
                            scratch[c] = make_int4( (int) out_h, (int) out_f, (int) out_s, 0 );
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

template <int R, int G>
static cudaError_t launch_one( const FastParams & p, int grid, size_t smem, cudaStream_t st ) {
    cudaError_t e = cudaFuncSetAttribute( sw_fast_kernel<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) smem );
    if( e != cudaSuccess )
        return e;
    sw_fast_kernel<R, G><<<grid, 256, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_sw_fast( int R, int G, const FastParams & p, int grid, cudaStream_t st ) {
    const size_t smem = 32ull * p.rows;
#define SSA_FAST_CASE( RR, GG ) \
    if( R == RR && G == GG ) \
        return launch_one<RR, GG>( p, grid, smem, st );
    SSA_FAST_CASE( 8, 8 )
    SSA_FAST_CASE( 16, 8 )
    SSA_FAST_CASE( 24, 8 )
    SSA_FAST_CASE( 32, 8 )
    SSA_FAST_CASE( 8, 16 )
    SSA_FAST_CASE( 16, 16 )
    SSA_FAST_CASE( 24, 16 )
    SSA_FAST_CASE( 32, 16 )
    SSA_FAST_CASE( 8, 32 )
    SSA_FAST_CASE( 16, 32 )
    SSA_FAST_CASE( 24, 32 )
    SSA_FAST_CASE( 32, 32 )
#undef SSA_FAST_CASE
    return cudaErrorInvalidValue;
}

// prof8[slot][code][row]: the query's 8-bit scores, -128 past the query and for
// the neutral pad code used after a sequence's last 4-column block.
__global__ void build_profile8_kernel( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * slots, uint32_t n, uint32_t rows, const int64_t * matrix, int8_t * prof,
        const uint64_t * prof_off ) {
    const uint32_t i = blockIdx.y;
    if( i >= n )
        return;
    const uint32_t slot = slots[i];
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
        const uint32_t * slots, uint32_t n, uint32_t rows, const int64_t * matrix, int8_t * prof,
        const uint64_t * prof_off, cudaStream_t st ) {
    if( n == 0 )
        return cudaSuccess;
    dim3 grid( 32, n );
    build_profile8_kernel<<<grid, 256, 0, st>>>( qcodes, qoff, qlen, slots, n, rows, matrix, prof, prof_off );
    return cudaGetLastError();
}

}  // namespace ssa
