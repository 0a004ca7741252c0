// noalloc.cu -- ssa_b200_score64_noalloc(): a database scoring call that
// allocates no memory.
//
// Who needs it: a caller that must not allocate device memory on its call
// path.  Two common cases are a serving process whose device memory is
// claimed up front by its own pool allocator (a cudaMalloc there either fails
// or takes memory the pool has promised elsewhere) and a latency-bound loop
// sharing the device with other streams (cudaFree synchronises the whole
// device, stalling every stream).  The regular search path sizes its device
// buffers to each request and grows them with cudaMalloc/cudaFree.
//
// What it computes: the Smith-Waterman or Needleman-Wunsch score of one query
// against every sequence of a database the caller already holds in device
// memory, as a BIT_WIDTH_64 search scores it (the library's 64-bit lane
// kernel, emul_kernel.cu at width 64).  Within this entry point's limits --
// query and sequences of at most 4096 residues, score-table entries within
// int16 (other tables are rejected), int8 gap penalties -- no value of the
// recurrence exceeds (4096 + 4096 + 8) x (32767 + 256) < 2^29 in magnitude,
// so int32 arithmetic and int32 scores give the 64-bit results exactly.
//
// Where its memory comes from: the file-scope __device__ arrays below, sized
// for the SSA_B200_NOALLOC_* limits of libssa_b200.h.  The CUDA driver reserves
// them when this file's module is loaded onto a device.  The first call on
// each device (with that device current) loads the module, looks up the
// arrays' addresses with cudaGetSymbolAddress and loads every kernel a call
// launches (CUDA loads modules lazily by default, and a load can allocate); a
// caller should make that first call before it enters its no-allocation phase
// (and before any stream capture).  Every later call only launches kernels
// and reads back one status word.  What must start at zero on every call (the
// work counter, the error word, the re-queue counter) is cleared by the call's
// first kernel.
//
// The addresses are looked up once per device ordinal in the device's primary
// context, the one the CUDA runtime uses: calls must be made with that context
// current (a context created through the driver API has its own copies of the
// arrays at other addresses).
//
// The arrays are shared by all calls on a device: two calls in flight on the
// same device at the same time (from two host threads, or on two streams)
// race on them and may return wrong scores.  Calls from one thread follow one
// another safely because each call waits for its own kernels.
#include "device_common.cuh"
#include "ssa_internal.h"
#include "libssa_b200.h"

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <mutex>

namespace ssa {

constexpr uint32_t NA_MAX_QUERY = SSA_B200_NOALLOC_MAX_QUERY;
constexpr uint32_t NA_MAX_SEQ_LEN = SSA_B200_NOALLOC_MAX_SEQ_LEN;
constexpr uint32_t NA_MAX_SEQS = SSA_B200_NOALLOC_MAX_SEQS;
constexpr int NA_BLOCKS = 16;                            // emulation kernel: 8 warps per block
constexpr uint32_t NA_WARPS = NA_BLOCKS * 8;
constexpr uint32_t NA_PROF_ROWS = (NA_MAX_QUERY + 255u) / 256u * 256u;   // query rows padded to a pass

// Scalars of a call.  counter, error_flags and next_count must be zero when
// the scoring kernel starts; the others describe the query as a one-slot
// batch (QueryView / the profile builder read them from device memory).
struct NoAllocState {
    unsigned long long counter;
    unsigned int error_flags;
    unsigned int next_count;
    uint64_t qoff;
    uint64_t prof_off;
    uint32_t qlen;
    uint32_t qpad;
};

static __device__ __align__( 256 ) int4 na_scratch[NA_WARPS * NA_MAX_SEQ_LEN];     // 8 MiB: pass boundary rows
static __device__ __align__( 256 ) int32_t na_profile[32 * NA_PROF_ROWS];         // 512 KiB: query profile
static __device__ __align__( 256 ) uint32_t na_order[NA_MAX_SEQS];                // 1 MiB: task -> sequence
static __device__ __align__( 256 ) int64_t na_matrix[1024];                       // substitution scores
static __device__ __align__( 256 ) NoAllocState na_state;

struct NoAllocDevice {
    bool ready = false;
    int4 * scratch = nullptr;
    int32_t * profile = nullptr;
    uint32_t * order = nullptr;
    int64_t * matrix = nullptr;
    NoAllocState * state = nullptr;
};

constexpr int NA_MAX_DEVICES = 64;
static NoAllocDevice na_devices[NA_MAX_DEVICES];
static std::mutex na_setup_mutex;

// The matrix travels as a kernel argument, so the call needs no host-to-device
// copy; int16 keeps the argument at 2 KiB (entries are checked on the host).
struct MatrixArg {
    int16_t v[1024];
};

__global__ void noalloc_prepare_kernel( MatrixArg m, uint32_t qlen, uint32_t qpad, uint32_t n_seqs ) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for( uint32_t i = tid; i < 1024u; i += stride )
        na_matrix[i] = m.v[i];
    for( uint32_t i = tid; i < n_seqs; i += stride )
        na_order[i] = i;
    if( tid == 0 ) {
        na_state.counter = 0;
        na_state.error_flags = 0;
        na_state.next_count = 0;
        na_state.qoff = 0;
        na_state.prof_off = 0;
        na_state.qlen = qlen;
        na_state.qpad = qpad;
    }
}

static int na_error( int code, const char * msg ) {
    fprintf( stderr, "ssa_b200_score64_noalloc: %s\n", msg );
    return code;
}

// Looks up the file-scope arrays of the current device once.
static int na_setup( int dev, NoAllocDevice ** out ) {
    std::lock_guard<std::mutex> lock( na_setup_mutex );
    NoAllocDevice & d = na_devices[dev];
    if( !d.ready ) {
        void * a[5] = {};
        if( cudaGetSymbolAddress( &a[0], na_scratch ) != cudaSuccess ||
                cudaGetSymbolAddress( &a[1], na_profile ) != cudaSuccess ||
                cudaGetSymbolAddress( &a[2], na_order ) != cudaSuccess ||
                cudaGetSymbolAddress( &a[3], na_matrix ) != cudaSuccess ||
                cudaGetSymbolAddress( &a[4], na_state ) != cudaSuccess )
            return na_error( SSA_B200_NOALLOC_ECUDA, cudaGetErrorString( cudaGetLastError() ) );
        // load every kernel a call launches now, not at its first launch
        cudaFuncAttributes fa;
        cudaError_t e = cudaFuncGetAttributes( &fa, noalloc_prepare_kernel );
        if( e == cudaSuccess )
            e = preload_emul64();
        if( e != cudaSuccess )
            return na_error( SSA_B200_NOALLOC_ECUDA, cudaGetErrorString( e ) );
        d.scratch = (int4 *) a[0];
        d.profile = (int32_t *) a[1];
        d.order = (uint32_t *) a[2];
        d.matrix = (int64_t *) a[3];
        d.state = (NoAllocState *) a[4];
        d.ready = true;
    }
    *out = &d;
    return SSA_B200_NOALLOC_OK;
}

}  // namespace ssa

#pragma GCC visibility push( default )
extern "C" int ssa_b200_score64_noalloc( int algorithm, const uint8_t * d_query, uint32_t query_len,
        const uint8_t * d_db_codes, const uint64_t * d_db_offsets, const uint32_t * d_db_lengths, uint32_t n_seqs,
        uint32_t max_seq_len, int32_t * d_scores, void * stream ) {
    using namespace ssa;
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH )
        return na_error( SSA_B200_NOALLOC_EINVAL, "algorithm must be SSA_SMITH_WATERMAN or SSA_NEEDLEMAN_WUNSCH" );
    if( query_len == 0 || !d_query || !d_db_codes || !d_db_offsets || !d_db_lengths || !d_scores )
        return na_error( SSA_B200_NOALLOC_EINVAL, "empty query or null device pointer" );
    if( query_len > NA_MAX_QUERY )
        return na_error( SSA_B200_NOALLOC_ETOOBIG, "query longer than SSA_B200_NOALLOC_MAX_QUERY (4096) residues" );
    if( max_seq_len > NA_MAX_SEQ_LEN )
        return na_error( SSA_B200_NOALLOC_ETOOBIG,
                "max_seq_len above SSA_B200_NOALLOC_MAX_SEQ_LEN (4096) residues" );
    if( n_seqs > NA_MAX_SEQS )
        return na_error( SSA_B200_NOALLOC_ETOOBIG, "more than SSA_B200_NOALLOC_MAX_SEQS (262144) sequences" );
    const Config & cfg = config();
    if( !cfg.matrix_set )
        return na_error( SSA_B200_NOALLOC_EINVAL, "no score matrix: call init_score_matrix or init_constant_scores" );
    MatrixArg m;
    for( int k = 0; k < 1024; k++ ) {
        if( cfg.matrix[k] < INT16_MIN || cfg.matrix[k] > INT16_MAX )
            return na_error( SSA_B200_NOALLOC_EINVAL, "score matrix entry outside the int16 range" );
        m.v[k] = (int16_t) cfg.matrix[k];
    }
    int dev = 0;
    if( cudaGetDevice( &dev ) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES )
        return na_error( SSA_B200_NOALLOC_ECUDA, "no usable current CUDA device" );
    NoAllocDevice * d = nullptr;
    if( int rc = na_setup( dev, &d ) )
        return rc;
    if( n_seqs == 0 )
        return SSA_B200_NOALLOC_OK;

    cudaStream_t st = (cudaStream_t) stream;
    const uint32_t qpad = (query_len + 255u) / 256u * 256u;
    const int prep_blocks = (int) std::min<uint32_t>( 1024u, (n_seqs + 255u) / 256u + 1u );
    noalloc_prepare_kernel<<<prep_blocks, 256, 0, st>>>( m, query_len, qpad, n_seqs );
    cudaError_t e = cudaGetLastError();
    NoAllocState * s = d->state;
    if( e == cudaSuccess )
        e = launch_build_profile32( d_query, &s->qoff, &s->qlen, &s->qpad, &s->prof_off, d->matrix, 64, d->profile,
                1, st );
    if( e == cudaSuccess ) {
        EmulParams p{};
        p.db = DbView{ d_db_codes, d_db_offsets, d_db_lengths, n_seqs };
        p.qv = QueryView{ d->profile, &s->prof_off, &s->qlen, &s->qpad, 1 };
        p.tasks = nullptr;
        p.order = d->order;
        p.slot_list = nullptr;
        p.n_sub = 0;
        p.n_tasks = n_seqs;
        p.counter = &s->counter;
        p.gap_open = cfg.gap_open;
        p.gap_extend = cfg.gap_extend;
        // 64-bit lanes never overflow, so nothing is re-queued (next_cap 0).
        p.sink = PassSink{ d_scores, n_seqs, nullptr, &s->next_count, 0, &s->error_flags };
        p.scratch = d->scratch;
        p.scratch_cols = NA_MAX_SEQ_LEN;
        e = launch_emul( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, 64, p, NA_BLOCKS, st );
    }
    unsigned int flags = 0;
    if( e == cudaSuccess )
        e = cudaMemcpyFromSymbolAsync( &flags, na_state, sizeof flags, offsetof( NoAllocState, error_flags ),
                cudaMemcpyDeviceToHost, st );
    if( e == cudaSuccess )
        e = cudaStreamSynchronize( st );
    if( e != cudaSuccess )
        return na_error( SSA_B200_NOALLOC_ECUDA, cudaGetErrorString( e ) );
    if( flags & ERR_SCRATCH_OVERFLOW )
        return na_error( SSA_B200_NOALLOC_ESEQLEN, "a database sequence is longer than SSA_B200_NOALLOC_MAX_SEQ_LEN (4096) residues" );
    if( flags )
        return na_error( SSA_B200_NOALLOC_ECUDA, "scoring kernel reported an error" );
    return SSA_B200_NOALLOC_OK;
}
#pragma GCC visibility pop
