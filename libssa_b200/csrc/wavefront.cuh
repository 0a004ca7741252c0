// wavefront.cuh -- helpers of the warp wavefront kernels (one warp per
// alignment, lane k owns a band of query rows and works on database column
// s - k at step s): staged database residues, the previous stripe's boundary
// row, and the work counter that hands out alignments largest first.
#pragma once

#include "device_common.cuh"

namespace ssa {

// The previous pass's boundary row is read by lane 0 one column per step; a
// warp stages it in shared memory 32 columns ahead so that the read is never
// a global-memory round trip on the step's critical path.
struct BoundaryPrefetch {
    int4 * tile;     // 32 entries of this warp
    int4 pf;
    __device__ void start( const int4 * scratch, uint32_t scratch_cols, uint32_t cols, bool active, int lane ) {
        pf = make_int4( 0, 0, 0, 0 );
        if( active && (uint32_t) lane < scratch_cols && (uint32_t) lane < cols )
            pf = scratch[lane];
    }
    __device__ void step( const int4 * scratch, uint32_t scratch_cols, uint32_t cols, bool active, uint32_t s,
            int lane ) {
        if( active && (s & 31u) == 0 ) {
            __syncwarp();
            tile[lane] = pf;
            __syncwarp();
            const uint32_t col = s + 32u + (uint32_t) lane;
            if( col < scratch_cols && col < cols )
                pf = scratch[col];
        }
    }
    __device__ int4 get( uint32_t s ) const { return tile[s & 31u]; }
};

// At step s lane k works on stream position s - k, so the warp needs the
// database residues of positions s - 31 .. s.  They are staged in a 64-entry
// ring in shared memory, each 32 positions loaded (one per lane) 32 steps
// before use, so no step waits on a global load.  Position x is database index
// x, or b_end - x for the reverse pass.
struct ResidueRing {
    uint8_t * ring;      // 64 entries of this warp
    uint8_t pf;          // this lane's residue for the next refill
    const uint8_t * b;
    int32_t n;           // positions 0 .. n - 1
    int32_t rev_end;     // -1: forward, else b_end of the reverse pass
    __device__ uint8_t fetch( int32_t x ) const {
        if( x < 0 || x >= n )
            return 0;
        return b[rev_end < 0 ? x : rev_end - x];
    }
    __device__ void start( int lane ) { pf = fetch( lane ); }
    __device__ void step( uint32_t s, int lane ) {
        if( (s & 31u) == 0 ) {
            __syncwarp();
            ring[(s + (uint32_t) lane) & 63u] = pf;
            __syncwarp();
            pf = fetch( (int32_t) s + 32 + lane );
        }
    }
    __device__ int get( uint32_t s, int lane ) const { return ring[(s - (uint32_t) lane) & 63u]; }
};

// Hits are handed out one per warp from a global counter, largest first (the
// host sorts them), so that the longest alignments start first.
__device__ __forceinline__ uint32_t next_hit( unsigned long long * counter, int lane ) {
    unsigned long long v = 0;
    if( lane == 0 )
        v = atomicAdd( counter, 1ull );
    return (uint32_t) __shfl_sync( 0xffffffffu, v, 0 );
}

}  // namespace ssa
