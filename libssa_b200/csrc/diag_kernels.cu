// diag_kernels.cu -- measured integer-pipe peak, the denominator of the
// search kernels' roofline.
//
// The Smith-Waterman / Needleman-Wunsch recurrence is integer add/max work
// (4 adds and 5 maxes per cell in the reference's ALIGNCORE,
// src/algo/simd/search_simd_sw.c:172-182), bound by the integer ALU pipe, not
// by HBM or tensor cores.  On sm_100 the packed 16x2 max, the fused 16x2
// add-max (__viaddmax_s16x2), the 3-way max and the byte permute all issue to
// the ALU pipe at 16 lanes per clock per SM sub-partition.  A fused add-max is
// the most work one ALU instruction does for the recurrence (two operations in
// each 16-bit half), so the pipe's ceiling is
//     measured __viaddmax_s16x2 warp instructions/s x 32 threads x 2 halves x 2.
// ssa_b200_int_peak() times eight interleaved chains whose every step reads
// another chain (x_i = max(x_i + c, x_{i+1})), so the compiler can neither
// fold nor drop any of them.
#include <cuda_runtime.h>
#include <cstdint>

namespace ssa {

constexpr int PEAK_ITERS = 4096;
constexpr int PEAK_CHAINS = 8;

__global__ void __launch_bounds__( 256 ) int_peak_kernel( unsigned * sink, unsigned seed ) {
    unsigned x[PEAK_CHAINS];
    const unsigned c = seed * 0x9e3779b9u;
#pragma unroll
    for( int i = 0; i < PEAK_CHAINS; i++ )
        x[i] = threadIdx.x * (i + 3) ^ seed;
    for( int it = 0; it < PEAK_ITERS; it++ ) {
#pragma unroll
        for( int i = 0; i < PEAK_CHAINS; i++ )
            x[i] = __viaddmax_s16x2( x[i], c, x[(i + 1) % PEAK_CHAINS] );
    }
    unsigned r = 0;
#pragma unroll
    for( int i = 0; i < PEAK_CHAINS; i++ )
        r ^= x[i];
    if( r == 0x9e3779b9u )
        sink[blockIdx.x] = r;
}

// Issue-rate probe of one SIMD-video / DPX intrinsic: eight interleaved chains
// x_i = op(x_i, x_{i+1}) (three-operand forms also read x_{i+2}), so nothing
// folds.  Timing the launch gives intrinsics per clock per SM; ncu's
// instruction counters of the same launch give instructions per intrinsic.
// OP: 0 __viaddmax_s16x2, 1 __vmaxs2, 2 __vimax3_s16x2, 3 __vaddss2,
//     4 __vsubss2, 5 __vaddss4, 6 __vmaxs4, 7 __vsubus4, 8 __vaddus4,
//     9 __vmaxu4, 10 __vadd4, 11 __vsub4, 12 max.f16x2, 13 32-bit integer add.
template <int OP>
__device__ __forceinline__ unsigned probe_op( unsigned a, unsigned b, unsigned c ) {
    if constexpr( OP == 0 ) return __viaddmax_s16x2( a, b, c );
    else if constexpr( OP == 1 ) return __vmaxs2( a, b );
    else if constexpr( OP == 2 ) return __vimax3_s16x2( a, b, c );
    else if constexpr( OP == 3 ) return __vaddss2( a, b );
    else if constexpr( OP == 4 ) return __vsubss2( a, b );
    else if constexpr( OP == 5 ) return __vaddss4( a, b );
    else if constexpr( OP == 6 ) return __vmaxs4( a, b );
    else if constexpr( OP == 7 ) return __vsubus4( a, b );
    else if constexpr( OP == 8 ) return __vaddus4( a, b );
    else if constexpr( OP == 9 ) return __vmaxu4( a, b );
    else if constexpr( OP == 10 ) return __vadd4( a, b );
    else if constexpr( OP == 11 ) return __vsub4( a, b );
    else if constexpr( OP == 12 ) {
        unsigned r;
        asm( "max.f16x2 %0, %1, %2;" : "=r"( r ) : "r"( a ), "r"( b ) );
        return r;
    }
    else return a + b;
}

constexpr int PROBE_OPS = 14;
constexpr int PROBE_ITERS = 1024;

template <int OP>
__global__ void __launch_bounds__( 256 ) simd_probe_kernel( unsigned * sink, unsigned seed ) {
    unsigned x[PEAK_CHAINS];
#pragma unroll
    for( int i = 0; i < PEAK_CHAINS; i++ )
        x[i] = (threadIdx.x * (i + 3)) ^ (seed * 0x9e3779b9u);
    for( int it = 0; it < PROBE_ITERS; it++ ) {
#pragma unroll
        for( int i = 0; i < PEAK_CHAINS; i++ )
            x[i] = probe_op<OP>( x[i], x[(i + 1) % PEAK_CHAINS], x[(i + 2) % PEAK_CHAINS] );
    }
    unsigned r = 0;
#pragma unroll
    for( int i = 0; i < PEAK_CHAINS; i++ )
        r ^= x[i];
    if( r == 0x9e3779b9u )
        sink[blockIdx.x] = r;
}

template <int OP>
static void launch_probe( int blocks, unsigned * sink, unsigned seed ) {
    simd_probe_kernel<OP><<<blocks, 256>>>( sink, seed );
}

typedef void (*ProbeLaunch)( int, unsigned *, unsigned );
static const ProbeLaunch probe_launch[PROBE_OPS] = {
    launch_probe<0>, launch_probe<1>, launch_probe<2>, launch_probe<3>, launch_probe<4>, launch_probe<5>,
    launch_probe<6>, launch_probe<7>, launch_probe<8>, launch_probe<9>, launch_probe<10>, launch_probe<11>,
    launch_probe<12>, launch_probe<13> };

}  // namespace ssa

#pragma GCC visibility push( default )
extern "C" int ssa_b200_simd_rate( int op, double * per_clock_per_sm ) {
    using namespace ssa;
    if( op < 0 || op >= PROBE_OPS || !per_clock_per_sm )
        return -1;
    int dev = 0;
    cudaDeviceProp prop;
    if( cudaGetDevice( &dev ) != cudaSuccess || cudaGetDeviceProperties( &prop, dev ) != cudaSuccess )
        return -1;
    const int blocks = prop.multiProcessorCount * 8;
    unsigned * sink = nullptr;
    if( cudaMalloc( &sink, blocks * sizeof(unsigned) ) != cudaSuccess )
        return -1;
    cudaEvent_t a, b;
    cudaEventCreate( &a );
    cudaEventCreate( &b );
    probe_launch[op]( blocks, sink, 1 );
    cudaEventRecord( a );
    const int reps = 5;
    for( int r = 0; r < reps; r++ )
        probe_launch[op]( blocks, sink, 2 + r );
    cudaEventRecord( b );
    cudaEventSynchronize( b );
    float ms = 0;
    cudaEventElapsedTime( &ms, a, b );
    cudaEventDestroy( a );
    cudaEventDestroy( b );
    cudaFree( sink );
    if( cudaGetLastError() != cudaSuccess || ms <= 0 )
        return -1;
    int clk_khz = 0;
    cudaDeviceGetAttribute( &clk_khz, cudaDevAttrClockRate, dev );
    const double intrinsics = (double) reps * blocks * (256.0 / 32.0) * PROBE_ITERS * PEAK_CHAINS;
    *per_clock_per_sm = intrinsics / (ms * 1e-3) / prop.multiProcessorCount / (clk_khz * 1e3);
    return 0;
}

extern "C" int ssa_b200_int_peak( double * lane_ops_per_second, double * instructions_per_clock_per_sm ) {
    using namespace ssa;
    int dev = 0;
    if( cudaGetDevice( &dev ) != cudaSuccess )
        return -1;
    cudaDeviceProp prop;
    if( cudaGetDeviceProperties( &prop, dev ) != cudaSuccess )
        return -1;
    const int blocks = prop.multiProcessorCount * 8;
    unsigned * sink = nullptr;
    if( cudaMalloc( &sink, blocks * sizeof(unsigned) ) != cudaSuccess )
        return -1;
    cudaEvent_t a, b;
    cudaEventCreate( &a );
    cudaEventCreate( &b );
    int_peak_kernel<<<blocks, 256>>>( sink, 1 );
    cudaEventRecord( a );
    const int reps = 10;
    for( int r = 0; r < reps; r++ )
        int_peak_kernel<<<blocks, 256>>>( sink, 2 + r );
    cudaEventRecord( b );
    cudaEventSynchronize( b );
    float ms = 0;
    cudaEventElapsedTime( &ms, a, b );
    cudaEventDestroy( a );
    cudaEventDestroy( b );
    cudaFree( sink );
    if( cudaGetLastError() != cudaSuccess || ms <= 0 )
        return -1;
    // warp instructions per launch: warps x iterations x chains
    const double inst = (double) reps * blocks * (256.0 / 32.0) * PEAK_ITERS * PEAK_CHAINS;
    const double per_s = inst / (ms * 1e-3);
    if( lane_ops_per_second )
        *lane_ops_per_second = per_s * 32.0 * 2.0 * 2.0;
    if( instructions_per_clock_per_sm ) {
        int clk_khz = 0;
        cudaDeviceGetAttribute( &clk_khz, cudaDevAttrClockRate, dev );
        *instructions_per_clock_per_sm = per_s / prop.multiProcessorCount / (clk_khz * 1e3);
    }
    return 0;
}
#pragma GCC visibility pop
