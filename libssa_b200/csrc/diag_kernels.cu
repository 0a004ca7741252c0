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

}  // namespace ssa

#pragma GCC visibility push( default )
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
