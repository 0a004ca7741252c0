// emul_kernel.cu -- exact emulation of one libssa SIMD lane per database
// sequence, at 8-bit, 16-bit or 64-bit semantics, for Smith-Waterman and
// Needleman-Wunsch.
//
// The CPU library scores each database sequence in one lane of a saturating
// int8/int16 vector kernel (reference: src/algo/simd/search_simd_sw.c:172-441,
// src/algo/simd/search_simd_nw.c:180-516) or with scalar int64 code
// (src/algo/64/smith_waterman_63.c:32-98, needleman_wunsch_64.c:32-98).  A
// lane's result does not depend on its neighbours, so here one warp computes
// one (query, sequence) pair with the lane's exact arithmetic: every add
// saturates at the pass width, the 8/16-bit boundary values are the
// reference's truncated and saturated chains, and the pad columns of the
// sequence's last 4-column block are scored with residue code 0.  The warp
// also reproduces the lane's overflow test at every block end and reports the
// number of blocks the lane spent on the sequence, which the host needs to
// replay the CPU channel schedule.
//
// Layout: warp lane k owns query rows [pass*256 + 8k, pass*256 + 8k + 8); the
// sequence streams through the warp as a wavefront (lane k works on column
// step-k), passing H, F and the column aggregates of its bottom row to lane
// k+1 by shuffle.  Queries longer than 256 rows take several passes; the last
// lane's bottom row of a pass is kept in a per-warp scratch row in global
// memory and read back by lane 0 in the next pass.
#include "device_common.cuh"

#include <climits>

namespace ssa {

constexpr int EMUL_R = 8;                  // query rows per lane
constexpr int EMUL_ROWS = 32 * EMUL_R;     // rows per pass

template <int W>
struct Width {
    static constexpr int64_t MIN = (W == 64) ? INT64_MIN / 4 : -(int64_t(1) << (W - 1));
    static constexpr int64_t MAX = (W == 64) ? INT64_MAX / 4 : (int64_t(1) << (W - 1)) - 1;
    template <typename V>
    __device__ __forceinline__ static V sat( V x ) {
        if constexpr( W == 64 ) {
            return x;
        }
        else {
            return min( max( x, (V) MIN ), (V) MAX );
        }
    }
    __device__ __forceinline__ static int64_t sat64( int64_t x ) {
        if constexpr( W == 64 ) {
            return x;
        }
        else {
            return x < MIN ? MIN : (x > MAX ? MAX : x);
        }
    }
    __device__ __forceinline__ static int64_t trunc( int64_t x ) {
        if constexpr( W == 8 )
            return (int8_t) x;
        else if constexpr( W == 16 )
            return (int16_t) x;
        else
            return x;
    }
};

// NW boundary values of the lane (reference: search_simd_nw.c:233-240,
// 445-453, 494-502; needleman_wunsch_64.c:39-52), exact in int64.
template <int W>
struct NwBounds {
    int64_t gO, gE, gOE;
    __device__ NwBounds( int go, int ge ) : gO( go ), gE( ge ) {
        gOE = Width<W>::trunc( (int64_t) go + ge );
    }
    // H(-1, j): the diagonal input of row 0 at column j + 1.
    __device__ __forceinline__ int64_t top_h( int64_t j ) const {
        int64_t col = j + 1;  // Hd(col)
        if( col == 0 )
            return 0;
        if constexpr( W == 64 ) {
            return gO + col * gE;
        }
        else {
            if( col <= 3 )
                return Width<W>::trunc( gO + col * gE );
            int64_t h3 = Width<W>::trunc( gO + 3 * gE );
            return Width<W>::sat64( h3 + (col - 3) * gE );
        }
    }
    // F entering row 0 at column c.
    __device__ __forceinline__ int64_t top_f( int64_t c ) const {
        if constexpr( W == 64 ) {
            return 2 * gO + (c + 2) * gE;
        }
        else {
            int64_t fd;
            if( c <= 3 )
                fd = Width<W>::trunc( gO + (c + 1) * gE );
            else
                fd = Width<W>::sat64( Width<W>::trunc( gO + 4 * gE ) + (c - 3) * gE );
            return Width<W>::sat64( fd + gOE );
        }
    }
    // H(i, -1) and E(i, -1).
    __device__ __forceinline__ int64_t left_h( int64_t i ) const {
        if constexpr( W == 64 )
            return gO + (i + 1) * gE;
        else
            return Width<W>::sat64( gOE + i * gE );
    }
    __device__ __forceinline__ int64_t left_e( int64_t i ) const {
        if constexpr( W == 64 )
            return 2 * gO + (i + 2) * gE;
        else
            return Width<W>::sat64( left_h( i ) + gOE );
    }
};

// A boundary-row column as it goes through shared and global memory: H, F and
// the column aggregates (max; min for NW) of the bottom row.
template <typename V>
struct BoundaryCol;
template <>
struct BoundaryCol<int32_t> {
    using type = int4;
    __device__ __forceinline__ static int4 make( int32_t h, int32_t f, int32_t a, int32_t b ) {
        return make_int4( h, f, a, b );
    }
};
template <>
struct BoundaryCol<int64_t> {
    using type = longlong4;
    __device__ __forceinline__ static longlong4 make( int64_t h, int64_t f, int64_t a, int64_t b ) {
        return make_longlong4( h, f, a, b );
    }
};

// V: the value type, int32_t at every width; int64_t for the 64-bit pass when
// the settings' values can leave the int32 range (the host decides; scores
// then go to p.sink.score64).  At 8 and 16 bits every value saturates to the
// width, so int32 holds them exactly.
template <int ALGO, int W, typename V>
__global__ void __launch_bounds__( 256 ) emul_kernel( EmulParams p ) {
    static_assert( sizeof(V) == 4 || W == 64, "int64 values only in the 64-bit pass" );
    constexpr bool SW = (ALGO == 0);
    constexpr bool WIDE = sizeof(V) == 8;
    constexpr int R = EMUL_R;
    using Col = typename BoundaryCol<V>::type;
    __shared__ Col tiles[8][32];   // previous pass's boundary row, 32 columns ahead
    const int lane = threadIdx.x & 31;
    Col * tile = tiles[threadIdx.x >> 5];
    const uint64_t warp_global = (blockIdx.x * (uint64_t) blockDim.x + threadIdx.x) >> 5;
    Col * scratch = reinterpret_cast<Col *>( p.scratch ) + warp_global * p.scratch_cols;

    // Scalar parameters at the pass width (reference: search_simd_sw.c:319-320,
    // search_simd_nw.c:360-373).
    const V gE = p.gap_extend;
    const V gOE = (V) Width<W>::trunc( (int64_t) p.gap_open + p.gap_extend );
    const int32_t thresh = (int32_t) Width<W>::trunc( Width<W>::MIN - p.gap_open - p.gap_extend - 1 );
    const NwBounds<W> nb( p.gap_open, p.gap_extend );
    // SW values are biased by MIN at 8/16 bits (the reference's -128/-32768 is
    // its zero); the 64-bit kernel is unbiased with an explicit floor at 0.
    const V SW_ZERO = (W == 64) ? (V) 0 : (V) Width<W>::MIN;
    constexpr V V_LOW = WIDE ? (V) LLONG_MIN : (V) INT_MIN;
    constexpr V V_HIGH = WIDE ? (V) LLONG_MAX : (V) INT_MAX;

    for( ;; ) {
        unsigned long long t = 0;
        if( lane == 0 )
            t = atomicAdd( p.counter, 1ull );
        t = __shfl_sync( 0xffffffffu, t, 0 );
        if( t >= p.n_tasks )
            break;
        uint32_t slot, id;
        if( p.tasks ) {
            slot = p.tasks[t].qslot;
            id = p.tasks[t].id;
        }
        else if( p.slot_list ) {
            slot = p.slot_list[t % p.n_sub];
            id = p.order[t / p.n_sub];
        }
        else {
            slot = (uint32_t) (t % p.qv.n_slots);
            id = p.order[t / p.qv.n_slots];
        }
        const uint32_t L = p.db.lens[id];
        const uint32_t Lb = (L + 3u) & ~3u;          // pad to the block end
        const uint8_t * dseq = p.db.codes + p.db.offsets[id];
        const uint32_t Q = p.qv.qlen[slot];
        const uint32_t qpad = p.qv.qpad[slot];
        const V * prof;
        if constexpr( WIDE )
            prof = p.qv.prof64 + p.qv.prof32_off[slot];
        else
            prof = p.qv.prof32 + p.qv.prof32_off[slot];
        const uint32_t passes = (Q + EMUL_ROWS - 1) / EMUL_ROWS;

        V s_run = SW ? SW_ZERO : (V) 0;              // last lane, final pass
        V blk_min = 0, blk_max = 0;
        int first_ovf = -1;
        V nw_score = 0;

        for( uint32_t pass = 0; pass < passes; pass++ ) {
            const bool final_pass = (pass + 1 == passes);
            const int64_t row0 = (int64_t) pass * EMUL_ROWS + lane * R;
            const int nvalid = (int) max( (int64_t) 0, min( (int64_t) R, (int64_t) Q - row0 ) );
            const int rstar = (int) ((int64_t) Q - 1 - row0);   // row Q-1 if in [0, R)

            V H[R], E[R];
#pragma unroll
            for( int r = 0; r < R; r++ ) {
                if constexpr( SW ) {
                    H[r] = SW_ZERO;
                    E[r] = SW_ZERO;
                }
                else {
                    H[r] = (V) nb.left_h( row0 + r );
                    E[r] = (V) nb.left_e( row0 + r );
                }
            }
            V diag;
            if constexpr( SW )
                diag = SW_ZERO;
            else
                diag = (row0 == 0) ? (V) 0 : (V) nb.left_h( row0 - 1 );

            V out_h = 0, out_f = 0, out_a = 0, out_b = 0;
            Col pf = BoundaryCol<V>::make( 0, 0, 0, 0 );
            if( pass > 0 && (uint32_t) lane < p.scratch_cols && (uint32_t) lane < Lb )
                pf = scratch[lane];
            const uint32_t steps = Lb + 31;
            for( uint32_t s = 0; s < steps; s++ ) {
                if( pass > 0 && (s & 31u) == 0 ) {
                    __syncwarp();
                    tile[lane] = pf;
                    __syncwarp();
                    const uint32_t col = s + 32u + (uint32_t) lane;
                    if( col < p.scratch_cols && col < Lb )
                        pf = scratch[col];
                }
                V up_h = __shfl_up_sync( 0xffffffffu, out_h, 1 );
                V up_f = __shfl_up_sync( 0xffffffffu, out_f, 1 );
                V up_a = __shfl_up_sync( 0xffffffffu, out_a, 1 );
                V up_b = __shfl_up_sync( 0xffffffffu, out_b, 1 );
                const int64_t c = (int64_t) s - lane;
                if( c < 0 || c >= (int64_t) Lb )
                    continue;
                if( lane == 0 ) {
                    if( pass == 0 ) {
                        if constexpr( SW ) {
                            up_h = SW_ZERO;
                            up_f = SW_ZERO;
                            up_a = SW_ZERO;
                        }
                        else {
                            up_h = (V) nb.top_h( c );
                            up_f = (V) nb.top_f( c );
                            up_a = 0;     // column max  (identity: block check also uses 0)
                            up_b = 0;     // column min
                        }
                    }
                    else {
                        const Col v = tile[s & 31u];
                        up_h = v.x;
                        up_f = v.y;
                        up_a = v.z;
                        up_b = v.w;
                    }
                }
                const int d = (c < (int64_t) L) ? dseq[c] : 0;
                const V * pr = prof + (uint64_t) d * qpad + row0;
                V v[R];
#pragma unroll
                for( int r = 0; r < R; r += 4 ) {
                    if constexpr( WIDE ) {
                        const longlong2 x0 = *reinterpret_cast<const longlong2 *>( pr + r );
                        const longlong2 x1 = *reinterpret_cast<const longlong2 *>( pr + r + 2 );
                        v[r] = x0.x;
                        v[r + 1] = x0.y;
                        v[r + 2] = x1.x;
                        v[r + 3] = x1.y;
                    }
                    else {
                        const int4 x = *reinterpret_cast<const int4 *>( pr + r );
                        v[r] = x.x;
                        v[r + 1] = x.y;
                        v[r + 2] = x.z;
                        v[r + 3] = x.w;
                    }
                }
                V f = up_f;
                V hd = diag;
                V cmax = SW ? SW_ZERO : V_LOW, cmin = V_HIGH;
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    V x;
                    if constexpr( SW && W == 64 ) {
                        // full_sw: max(hdiag + s, e, f, 0)
                        x = max( max( hd + v[r], E[r] ), max( f, (V) 0 ) );
                    }
                    else {
                        // ALIGNCORE: H = sat(Hdiag + V); H = max(H, F); H = max(H, E)
                        x = max( max( Width<W>::sat( hd + v[r] ), f ), E[r] );
                    }
                    if( r < nvalid ) {
                        cmax = max( cmax, x );
                        cmin = min( cmin, x );
                    }
                    if constexpr( !SW ) {
                        if( r == rstar && c == (int64_t) L - 1 )
                            nw_score = x;
                    }
                    hd = H[r];
                    H[r] = x;
                    V y = Width<W>::sat( x + gOE );
                    f = max( Width<W>::sat( f + gE ), y );
                    E[r] = max( Width<W>::sat( E[r] + gE ), y );
                }
                diag = up_h;
                out_h = H[R - 1];
                out_f = f;
                if constexpr( SW ) {
                    out_a = max( up_a, cmax );
                }
                else {
                    out_a = max( up_a, cmax );
                    out_b = min( up_b, cmin );
                }
                if( lane == 31 ) {
                    if( !final_pass ) {
                        if( (uint32_t) c < p.scratch_cols )
                            scratch[c] = BoundaryCol<V>::make( out_h, out_f, out_a, out_b );
                        else
                            atomicOr( p.sink.error_flags, ERR_SCRATCH_OVERFLOW );
                    }
                    else if( first_ovf < 0 ) {
                        if constexpr( SW ) {
                            s_run = max( s_run, out_a );
                            if( (c & 3) == 3 && W != 64 && s_run == (V) Width<W>::MAX )
                                first_ovf = (int) (c >> 2);
                        }
                        else {
                            blk_max = max( blk_max, out_a );
                            blk_min = min( blk_min, out_b );
                            if( (c & 3) == 3 ) {
                                if( W != 64 && (blk_min < (V) thresh || blk_max == (V) Width<W>::MAX) )
                                    first_ovf = (int) (c >> 2);
                                blk_min = 0;
                                blk_max = 0;
                            }
                        }
                    }
                }
            }
            __syncwarp();
        }

        // Collect the lane's report.
        if constexpr( !SW ) {
            const int owner = (int) (((int64_t) Q - 1 - (int64_t) (passes - 1) * EMUL_ROWS) / R);
            nw_score = __shfl_sync( 0xffffffffu, nw_score, owner );
        }
        if( lane == 31 ) {
            V score;
            bool ok;
            if constexpr( SW ) {
                score = (W == 64) ? s_run : (V) (s_run - (V) Width<W>::MIN);
                ok = first_ovf < 0 && (W == 64 || (int64_t) score < ((int64_t) 1 << W) - 1);
            }
            else {
                score = nw_score;
                ok = first_ovf < 0 && (W == 64 || (score > (V) Width<W>::MIN && score < (V) Width<W>::MAX));
            }
            const int32_t nblocks = first_ovf >= 0 ? first_ovf + 1 : (int32_t) (Lb >> 2);
            const uint64_t at = (uint64_t) slot * p.sink.score_stride + id;
            if constexpr( WIDE ) {
                p.sink.score64[at] = score;
                if( p.sink.score )
                    p.sink.score[at] = SCORE_IN_WIDE;
            }
            else {
                p.sink.score[at] = score;
            }
            if( !ok ) {
                unsigned k = atomicAdd( p.sink.next_count, 1u );
                if( k < p.sink.next_cap )
                    p.sink.next[k] = PairTask{ slot, id, nblocks, 0 };
                else
                    atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
            }
        }
        __syncwarp();
    }
}

// Host-side launcher.
cudaError_t launch_emul( int algo, int width, const EmulParams & p, int grid, cudaStream_t st, bool wide ) {
    dim3 block( 256 );
    if( wide ) {
        if( width != 64 || !p.qv.prof64 || !p.sink.score64 )
            return cudaErrorInvalidValue;
        if( algo == 0 )
            emul_kernel<0, 64, int64_t><<<grid, block, 0, st>>>( p );
        else
            emul_kernel<1, 64, int64_t><<<grid, block, 0, st>>>( p );
        return cudaGetLastError();
    }
#define SSA_EMUL_CASE( A, Wd ) \
    if( algo == A && width == Wd ) { \
        emul_kernel<A, Wd, int32_t><<<grid, block, 0, st>>>( p ); \
        return cudaGetLastError(); \
    }
    SSA_EMUL_CASE( 0, 8 )
    SSA_EMUL_CASE( 0, 16 )
    SSA_EMUL_CASE( 0, 64 )
    SSA_EMUL_CASE( 1, 8 )
    SSA_EMUL_CASE( 1, 16 )
    SSA_EMUL_CASE( 1, 64 )
#undef SSA_EMUL_CASE
    return cudaErrorInvalidValue;
}

// prof32[slot][code][row] = matrix[(code << 5) + query[row]] at the pass width;
// rows past the query are 0 (they never reach a result).
__global__ void build_profile32_kernel( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int width, int32_t * prof,
        uint32_t n_slots ) {
    const uint32_t slot = blockIdx.y;
    if( slot >= n_slots )
        return;
    const uint32_t Q = qlen[slot], P = qpad[slot];
    const uint8_t * q = qcodes + qoff[slot];
    int32_t * out = prof + prof_off[slot];
    for( uint64_t k = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; k < 32ull * P;
            k += (uint64_t) gridDim.x * blockDim.x ) {
        uint32_t code = (uint32_t) (k / P), row = (uint32_t) (k % P);
        int32_t v = 0;
        if( row < Q ) {
            int64_t m = matrix[(code << 5) + q[row]];
            v = (width == 8) ? (int32_t) (int8_t) m : (width == 16) ? (int32_t) (int16_t) m : (int32_t) m;
        }
        out[k] = v;
    }
}

cudaError_t launch_build_profile32( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int width, int32_t * prof,
        uint32_t n_slots, cudaStream_t st ) {
    dim3 grid( 64, n_slots );
    build_profile32_kernel<<<grid, 256, 0, st>>>( qcodes, qoff, qlen, qpad, prof_off, matrix, width, prof, n_slots );
    return cudaGetLastError();
}

// prof64[slot][code][row] = matrix[(code << 5) + query[row]], exact; rows
// past the query are 0.
__global__ void build_profile64_kernel( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int64_t * prof,
        uint32_t n_slots ) {
    const uint32_t slot = blockIdx.y;
    if( slot >= n_slots )
        return;
    const uint32_t Q = qlen[slot], P = qpad[slot];
    const uint8_t * q = qcodes + qoff[slot];
    int64_t * out = prof + prof_off[slot];
    for( uint64_t k = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; k < 32ull * P;
            k += (uint64_t) gridDim.x * blockDim.x ) {
        const uint32_t code = (uint32_t) (k / P), row = (uint32_t) (k % P);
        out[k] = (row < Q) ? matrix[(code << 5) + q[row]] : 0;
    }
}

// Loads the int32 64-bit lane kernels and the int32 profile builder onto the
// current device now: under lazy module loading (the CUDA default) a kernel
// is loaded, which can allocate device memory, at its first launch otherwise.
cudaError_t preload_emul64() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes( &a, emul_kernel<0, 64, int32_t> );
    if( e == cudaSuccess )
        e = cudaFuncGetAttributes( &a, emul_kernel<1, 64, int32_t> );
    if( e == cudaSuccess )
        e = cudaFuncGetAttributes( &a, build_profile32_kernel );
    return e;
}

cudaError_t launch_build_profile64( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qpad, const uint64_t * prof_off, const int64_t * matrix, int64_t * prof, uint32_t n_slots,
        cudaStream_t st ) {
    dim3 grid( 64, n_slots );
    build_profile64_kernel<<<grid, 256, 0, st>>>( qcodes, qoff, qlen, qpad, prof_off, matrix, prof, n_slots );
    return cudaGetLastError();
}

}  // namespace ssa
