// sw_qpair_kernel.cu -- the Smith-Waterman 8-bit-entry search pass for
// batches: two queries per register.
//
// Semantics are those of sw_fast_kernel.cu (exact 16-bit scores with a +1024
// bias per half, the first column at which a running maximum reaches 255
// gives the reference lane's overflow block; reference:
// src/algo/simd/search_simd_sw.c:172-182, 369-382, 422-423).  What changes is
// what shares a register: here the low half carries query A and the high half
// query B of a length-sorted query pair, both against the same database
// sequence.  The profile word of a (residue, row) is then one 16x2 value that
// a 128-bit shared load delivers four rows at a time, so the cell update needs
// no byte permute, and each database residue is read once for two queries.
//
// Mapping onto sm_100:
//   * a group of QP_G = 4 threads computes one database sequence as a
//     wavefront, thread k owning R query rows of the current pass in
//     registers; eight groups (eight sequences of similar length) fill a warp;
//   * a thread advances two columns per step and interleaves them row by row
//     (cell (r, c) then cell (r - 1, c + 1)), which gives two independent
//     dependency chains and lets H be updated in place without copies;
//   * per 16x2 cell pair: one 3-way max, three fused add-max (ALU pipe), one
//     IADD, and half a 3-way max for the running maximum;
//   * H and F of the bottom rows of both columns go to thread k + 1 by
//     shuffle; the running maximum is kept per thread and combined over the
//     group only at the end of the sequence, together with the first column
//     pair at which each thread's maximum reached 255;
//   * queries longer than QP_G x R rows take several passes over a sequence;
//     the bottom row's H and F go through a per-group scratch row in global
//     memory, read back by thread 0 two steps ahead;
//   * every warp schedules itself: (query pair, range of sequences) units from
//     a global counter, the longest query pairs first so that the last units
//     to start are short ones; the warp's shared-memory slice holds the
//     current pass's rows of the query pair's profile.
#include "device_common.cuh"

#include <climits>

namespace ssa {

constexpr uint32_t QP_BIAS = 1024u;
constexpr uint32_t QP_BIAS2 = (QP_BIAS << 16) | QP_BIAS;
// adding this per half sets bit 15 exactly when the half is >= 1024 + 255
// (halves stay in [0, 32767], so no carry crosses into the other half)
constexpr uint32_t QP_CROSS_ADD = ((0x8000u - (QP_BIAS + 255u)) << 16) | (0x8000u - (QP_BIAS + 255u));
constexpr int QP_THREADS = QP_THREADS_PER_CTA;

// MB: resident CTAs per SM the register allocation is bounded for (4: up to
// 128 registers a thread, 5: up to 102); chosen per class by the tuning table.
template <int R, int MB>
__global__ void __launch_bounds__( QP_THREADS, MB ) sw_qpair_kernel( QPairParams p ) {
    constexpr int G = QP_G;
    constexpr uint32_t GR = (uint32_t) (G * R);
    extern __shared__ __align__( 16 ) uint32_t qsm[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t * slice = qsm + warp_in_cta * (QP_CODES * GR);
    const int k = lane & (G - 1);                // thread within its group
    const int g = lane / G;                      // group within the warp
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) p.gap_e << 16) | (uint16_t) (int16_t) p.gap_e;
    int4 * scratch = p.scratch + ((uint64_t) warp_global * QP_GPW + (uint32_t) g) * p.scratch_cols;
    uint64_t loaded_key = ~0ull;

    for( ;; ) {
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t qp = p.unit_pairs[u / p.n_chunks];
        const uint32_t chunk = (uint32_t) (u % p.n_chunks);
        const uint32_t seq_begin = p.chunk_bounds[chunk], seq_end = p.chunk_bounds[chunk + 1];
        const uint32_t rows = p.qp_rows[qp];
        const uint32_t passes = rows / GR;
        const uint32_t * prof = p.prof + p.prof_off[qp];
        const uint32_t slot_a = p.qp_slots[2 * qp], slot_b = p.qp_slots[2 * qp + 1];

        for( uint32_t b0 = seq_begin; b0 < seq_end; b0 += (uint32_t) QP_GPW ) {
            const uint32_t idx = b0 + (uint32_t) g;
            const bool valid = idx < seq_end;
            const uint32_t id = valid ? p.order[idx] : 0u;
            const uint32_t L = valid ? p.db.lens[id] : 0u;
            const uint32_t ncp = ((L + 3u) & ~3u) >> 1;          // column pairs up to the block end
            const uint32_t max_ncp = __reduce_max_sync( 0xffffffffu, ncp );
            const uint8_t * res = p.db.codes + (valid ? p.db.offsets[id] : 0ull);

            // per thread over all passes: running maximum and the first column
            // pair at which it reached 255 (per half)
            uint32_t best = QP_BIAS2;
            int cross_a = INT_MAX, cross_b = INT_MAX;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool last_pass = (pass + 1 == passes);
                const uint64_t key = ((uint64_t) qp << 24) | pass;
                if( key != loaded_key ) {
                    // this pass's rows of all residue codes: QP_CODES x GR words
                    __syncwarp();
                    constexpr uint32_t per_code = GR / 4u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < QP_CODES * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 4u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = QP_BIAS2;
                    E[r] = QP_BIAS2;
                }
                uint32_t diag = QP_BIAS2, smax = QP_BIAS2, seen = 0;
                uint32_t out_h0 = QP_BIAS2, out_f0 = QP_BIAS2, out_h1 = QP_BIAS2, out_f1 = QP_BIAS2;
                // residues of column pairs cp .. cp + 3 (two codes each), one pair
                // fetched ahead every step; past the block end the reads stay
                // inside the padded record or the next one (never used)
                const uint32_t fetch_limit = ncp + 3u;
                auto fetch = [&]( int32_t cp ) -> uint32_t {
                    const uint32_t c = min( (uint32_t) max( cp, 0 ), fetch_limit );
                    return (uint32_t) *reinterpret_cast<const uint16_t *>( res + 2u * c );
                };
                uint32_t q0 = fetch( -k ), q1 = fetch( 1 - k ), q2 = fetch( 2 - k ), q3 = fetch( 3 - k );
                // thread 0: the previous pass's bottom row, two column pairs ahead
                const bool reads_boundary = (k == 0) && pass > 0;
                int4 bq0 = make_int4( 0, 0, 0, 0 ), bq1 = bq0;
                if( reads_boundary ) {
                    if( ncp > 0 )
                        bq0 = scratch[0];
                    if( ncp > 1 )
                        bq1 = scratch[1];
                }
                const uint32_t steps = max_ncp + (uint32_t) G - 1u;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h0 = __shfl_up_sync( 0xffffffffu, out_h0, 1, G );
                    uint32_t up_f0 = __shfl_up_sync( 0xffffffffu, out_f0, 1, G );
                    uint32_t up_h1 = __shfl_up_sync( 0xffffffffu, out_h1, 1, G );
                    uint32_t up_f1 = __shfl_up_sync( 0xffffffffu, out_f1, 1, G );
                    const int32_t cp = (int32_t) s - k;
                    const uint32_t w = q0;
                    q0 = q1;
                    q1 = q2;
                    q2 = q3;
                    q3 = fetch( cp + 4 );
                    const int4 bnd = bq0;
                    if( reads_boundary ) {
                        bq0 = bq1;
                        const uint32_t nxt = (uint32_t) cp + 2u;
                        if( nxt < ncp && nxt < p.scratch_cols )
                            bq1 = scratch[nxt];
                    }
                    if( cp < 0 || (uint32_t) cp >= ncp )
                        continue;
                    if( k == 0 ) {
                        up_h0 = pass ? (uint32_t) bnd.x : QP_BIAS2;
                        up_f0 = pass ? (uint32_t) bnd.y : QP_BIAS2;
                        up_h1 = pass ? (uint32_t) bnd.z : QP_BIAS2;
                        up_f1 = pass ? (uint32_t) bnd.w : QP_BIAS2;
                    }
                    const uint32_t * pa = slice + (w & 0xffu) * GR + (uint32_t) (k * R);
                    const uint32_t * pb = slice + (w >> 8) * GR + (uint32_t) (k * R);
                    // profile words four rows at a time, loaded as the rows come up
                    uint4 xa = make_uint4( 0, 0, 0, 0 ), xb = xa;
                    // column c = 2cp (cell A, row r) interleaved with column
                    // c + 1 (cell B, row r - 1); H[r] keeps column c - 1 until
                    // cell B of row r overwrites it with column c + 1
                    uint32_t fa = up_f0, fb = up_f1;
                    uint32_t hc_prev = 0, hc_prev2 = 0;     // column c, rows r - 1 and r - 2
#pragma unroll
                    for( int r = 0; r <= R; r++ ) {
                        uint32_t ha = 0;
                        if( r < R ) {
                            if( (r & 3) == 0 )
                                xa = *reinterpret_cast<const uint4 *>( pa + r );
                            const uint32_t v = (r & 3) == 0 ? xa.x : (r & 3) == 1 ? xa.y : (r & 3) == 2 ? xa.z : xa.w;
                            const uint32_t hd = (r == 0) ? diag : H[r - 1];
                            const uint32_t t = __vimax3_s16x2( E[r], fa, QP_BIAS2 );
                            ha = __viaddmax_s16x2( hd, v, t );
                            const uint32_t hg = ha + GOE32;
                            fa = __viaddmax_s16x2( fa, GE2, hg );
                            E[r] = __viaddmax_s16x2( E[r], GE2, hg );
                        }
                        if( r >= 1 ) {
                            const int rb = r - 1;
                            if( (rb & 3) == 0 )
                                xb = *reinterpret_cast<const uint4 *>( pb + rb );
                            const uint32_t v = (rb & 3) == 0 ? xb.x : (rb & 3) == 1 ? xb.y : (rb & 3) == 2 ? xb.z : xb.w;
                            const uint32_t hd = (rb == 0) ? up_h0 : hc_prev2;
                            const uint32_t t = __vimax3_s16x2( E[rb], fb, QP_BIAS2 );
                            const uint32_t hb = __viaddmax_s16x2( hd, v, t );
                            const uint32_t hg = hb + GOE32;
                            fb = __viaddmax_s16x2( fb, GE2, hg );
                            E[rb] = __viaddmax_s16x2( E[rb], GE2, hg );
                            H[rb] = hb;
                            smax = (r < R) ? __vimax3_s16x2( smax, ha, hb ) : __vmaxs2( smax, hb );
                        }
                        else {
                            smax = __vmaxs2( smax, ha );
                        }
                        hc_prev2 = hc_prev;
                        hc_prev = ha;
                    }
                    diag = up_h1;
                    out_h0 = hc_prev2;       // column c, row R - 1
                    out_f0 = fa;
                    out_h1 = H[R - 1];
                    out_f1 = fb;
                    // first column pair at which this thread's maximum reached 255
                    const uint32_t ge = (smax + QP_CROSS_ADD) & 0x80008000u;
                    if( ge != seen ) {
                        if( (ge & 0x8000u) && !(seen & 0x8000u) )
                            cross_a = min( cross_a, cp );
                        if( (ge & 0x80000000u) && !(seen & 0x80000000u) )
                            cross_b = min( cross_b, cp );
                        seen = ge;
                    }
                    if( k == G - 1 && !last_pass ) {
                        if( (uint32_t) cp < p.scratch_cols )
                            scratch[cp] = make_int4( (int) out_h0, (int) out_f0, (int) out_h1, (int) out_f1 );
                        else
                            atomicOr( p.sink.error_flags, ERR_SCRATCH_OVERFLOW );
                    }
                }
                best = __vmaxs2( best, smax );
                __syncwarp();
            }
            // combine the group's threads: maximum and earliest crossing
#pragma unroll
            for( int o = 1; o < G; o <<= 1 ) {
                best = __vmaxs2( best, __shfl_xor_sync( 0xffffffffu, best, o, G ) );
                cross_a = min( cross_a, __shfl_xor_sync( 0xffffffffu, cross_a, o, G ) );
                cross_b = min( cross_b, __shfl_xor_sync( 0xffffffffu, cross_b, o, G ) );
            }
            if( valid && k == 0 ) {
                const uint32_t slots[2] = { slot_a, slot_b };
                const int cross[2] = { cross_a, cross_b };
                const uint32_t sv[2] = { best & 0xffffu, best >> 16 };
#pragma unroll
                for( int h = 0; h < 2; h++ ) {
                    if( slots[h] == 0xffffffffu )
                        continue;
                    int32_t * dst = p.sink.score + (uint64_t) slots[h] * p.sink.score_stride + id;
                    if( cross[h] == INT_MAX ) {
                        *dst = (int32_t) (sv[h] - QP_BIAS);
                    }
                    else {
                        // columns 2cp and 2cp + 1 lie in 4-column block cp / 2
                        *dst = 255;
                        unsigned q = atomicAdd( p.sink.next_count, 1u );
                        if( q < p.sink.next_cap )
                            p.sink.next[q] = PairTask{ slots[h], id, (cross[h] >> 1) + 1, 0 };
                        else
                            atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same pass, one 4-column block per step: a thread interleaves four
// columns (cell (r, c + j) in row iteration r + j, j = 0..3), four independent
// dependency chains instead of two.  The semantics, the group layout, the
// profile slices and the scheduling are those of sw_qpair_kernel; a step reads
// one 32-bit word of residues (the block) and crosses the pass boundary as two
// int4 per block (H and F of the bottom row, four columns).  The running
// maximum's first crossing of 255 is recorded per block directly.
//
// H[r] holds column c - 1 (the previous step's last column) until chain 3
// overwrites it with column c + 3 (iteration r + 3); chain j reads the
// diagonal H(r - 1, c + j - 1) from chain j - 1's value two iterations back,
// and E[r] passes from chain j - 1 (iteration r + j - 1) to chain j.
// ---------------------------------------------------------------------------
// The running maximum of H as fp16x2: every H is at least the bias (1024, the
// fp16 bit pattern of a positive normal number), and positive fp16 values
// order like their bit patterns, so a half-precision max of the bit patterns
// is the integer max.  Patterns past 0x7c00 (infinity, NaN) -- scores more
// than 30,000 above the bias -- are ignored or taken as the largest; a cell
// only gets there through cells that crossed 255 earlier on its path, whose
// own crossing is recorded, so the first crossing and every reported score
// (below 255) are unchanged.  This max issues to another pipe than the
// integer ALU, which the rest of the recurrence saturates.
__device__ __forceinline__ uint32_t hmax_bits( uint32_t a, uint32_t b ) {
    uint32_t r;
    asm( "max.f16x2 %0, %1, %2;" : "=r"( r ) : "r"( a ), "r"( b ) );
    return r;
}

// The 4-column kernel loads database residues with the streaming cache
// operator (ld.global.cs: evict first): the database passes through L2 once
// per pass and query pair, and the pass-boundary row of a multi-pass query,
// written in one pass and read back in the next, should stay there instead.
// HM: track the running maximum with hmax_bits (one instruction per cell
// pair, off the ALU pipe) instead of the 3-way integer max (half an ALU
// instruction per cell pair).
// G: threads per database sequence (4, or 8 with R = 12: one group per
// quarter-warp, whose rows 12k fall into 8 distinct shared-memory bank groups,
// so the 128-bit profile loads are conflict-free; a pass still holds 96 rows).
template <int R, int MB, bool HM, int G = QP_G>
__global__ void __launch_bounds__( QP_THREADS, MB ) sw_qpair4_kernel( QPairParams p ) {
    static_assert( G == 4 || G == 8, "4 or 8 threads per sequence" );
    constexpr int GPW = 32 / G;                  // sequences per warp
    constexpr int C = 4;
    constexpr uint32_t GR = (uint32_t) (G * R);
    extern __shared__ __align__( 16 ) uint32_t qsm[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t * slice = qsm + warp_in_cta * (QP_CODES * GR);
    const int k = lane & (G - 1);
    const int g = lane / G;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) p.gap_e << 16) | (uint16_t) (int16_t) p.gap_e;
    int4 * scratch = p.scratch + ((uint64_t) warp_global * QP_GPW + (uint32_t) g) * p.scratch_cols;
    uint64_t loaded_key = ~0ull;

    for( ;; ) {
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t qp = p.unit_pairs[u / p.n_chunks];
        const uint32_t chunk = (uint32_t) (u % p.n_chunks);
        const uint32_t seq_begin = p.chunk_bounds[chunk], seq_end = p.chunk_bounds[chunk + 1];
        const uint32_t rows = p.qp_rows[qp];
        const uint32_t passes = rows / GR;
        const uint32_t * prof = p.prof + p.prof_off[qp];
        const uint32_t slot_a = p.qp_slots[2 * qp], slot_b = p.qp_slots[2 * qp + 1];

        for( uint32_t b0 = seq_begin; b0 < seq_end; b0 += (uint32_t) GPW ) {
            const uint32_t idx = b0 + (uint32_t) g;
            const bool valid = idx < seq_end;
            const uint32_t id = valid ? p.order[idx] : 0u;
            const uint32_t L = valid ? p.db.lens[id] : 0u;
            const uint32_t nb = (L + 3u) >> 2;                    // 4-column blocks
            const uint32_t max_nb = __reduce_max_sync( 0xffffffffu, nb );
            const uint8_t * res = p.db.codes + (valid ? p.db.offsets[id] : 0ull);

            uint32_t best = QP_BIAS2;
            int cross_a = INT_MAX, cross_b = INT_MAX;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool last_pass = (pass + 1 == passes);
                const uint64_t key = ((uint64_t) qp << 24) | pass;
                if( key != loaded_key ) {
                    __syncwarp();
                    constexpr uint32_t per_code = GR / 4u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < QP_CODES * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 4u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = QP_BIAS2;
                    E[r] = QP_BIAS2;
                }
                uint32_t diag = QP_BIAS2, smax = QP_BIAS2, seen = 0;
                uint32_t out_h[C], out_f[C];
#pragma unroll
                for( int j = 0; j < C; j++ ) {
                    out_h[j] = QP_BIAS2;
                    out_f[j] = QP_BIAS2;
                }
                // residues of blocks b .. b + 3, one block fetched ahead every
                // step; past the last block the reads stay inside the padded
                // record or the next one (never used)
                const uint32_t fetch_limit = nb + 3u;
                auto fetch = [&]( int32_t b ) -> uint32_t {
                    const uint32_t c = min( (uint32_t) max( b, 0 ), fetch_limit );
                    return __ldcs( reinterpret_cast<const unsigned int *>( res + 4u * c ) );
                };
                uint32_t q0 = fetch( -k ), q1 = fetch( 1 - k ), q2 = fetch( 2 - k ), q3 = fetch( 3 - k );
                // thread 0: the previous pass's bottom row, one block ahead
                const bool reads_boundary = (k == 0) && pass > 0;
                int4 bq0 = make_int4( 0, 0, 0, 0 ), bq1 = bq0;
                if( reads_boundary && nb > 0 ) {
                    bq0 = scratch[0];
                    bq1 = scratch[1];
                }
                const uint32_t steps = max_nb + (uint32_t) G - 1u;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h[C], up_f[C];
#pragma unroll
                    for( int j = 0; j < C; j++ ) {
                        up_h[j] = __shfl_up_sync( 0xffffffffu, out_h[j], 1, G );
                        up_f[j] = __shfl_up_sync( 0xffffffffu, out_f[j], 1, G );
                    }
                    const int32_t b = (int32_t) s - k;
                    const uint32_t w = q0;
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
                                up_h[j] = QP_BIAS2;
                                up_f[j] = QP_BIAS2;
                            }
                        }
                    }
                    const uint32_t * pc[C];
#pragma unroll
                    for( int j = 0; j < C; j++ )
                        pc[j] = slice + ((w >> (8 * j)) & 0xffu) * GR + (uint32_t) (k * R);
                    uint4 x[C];
                    uint32_t f[C];
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
                            if( (r & 3) == 0 )
                                x[j] = *reinterpret_cast<const uint4 *>( pc[j] + r );
                            const uint32_t v = (r & 3) == 0 ? x[j].x : (r & 3) == 1 ? x[j].y
                                    : (r & 3) == 2 ? x[j].z : x[j].w;
                            uint32_t hd;
                            if( r == 0 )
                                hd = (j == 0) ? diag : up_h[j - 1];
                            else
                                hd = (j == 0) ? H[r - 1] : hv[j - 1][r - 1];
                            const uint32_t t = __vimax3_s16x2( E[r], f[j], QP_BIAS2 );
                            const uint32_t h = __viaddmax_s16x2( hd, v, t );
                            const uint32_t hg = h + GOE32;
                            f[j] = __viaddmax_s16x2( f[j], GE2, hg );
                            E[r] = __viaddmax_s16x2( E[r], GE2, hg );
                            hv[j][r] = h;
                            hnew[j] = h;
                        }
                        // the new cells of this iteration into the running maximum
                        const int j0 = it - (R - 1) > 0 ? it - (R - 1) : 0;
                        const int j1 = it < C - 1 ? it : C - 1;
                        if constexpr( HM ) {
#pragma unroll
                            for( int j = j0; j <= j1; j++ )
                                smax = hmax_bits( smax, hnew[j] );
                        }
                        else {
#pragma unroll
                            for( int j = j0; j <= j1; j += 2 ) {
                                if( j + 1 <= j1 )
                                    smax = __vimax3_s16x2( smax, hnew[j], hnew[j + 1] );
                                else
                                    smax = __vmaxs2( smax, hnew[j] );
                            }
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
                    const uint32_t ge = (smax + QP_CROSS_ADD) & 0x80008000u;
                    if( ge != seen ) {
                        if( (ge & 0x8000u) && !(seen & 0x8000u) )
                            cross_a = min( cross_a, b );
                        if( (ge & 0x80000000u) && !(seen & 0x80000000u) )
                            cross_b = min( cross_b, b );
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
#pragma unroll
            for( int o = 1; o < G; o <<= 1 ) {
                best = __vmaxs2( best, __shfl_xor_sync( 0xffffffffu, best, o, G ) );
                cross_a = min( cross_a, __shfl_xor_sync( 0xffffffffu, cross_a, o, G ) );
                cross_b = min( cross_b, __shfl_xor_sync( 0xffffffffu, cross_b, o, G ) );
            }
            if( valid && k == 0 ) {
                const uint32_t slots[2] = { slot_a, slot_b };
                const int cross[2] = { cross_a, cross_b };
                const uint32_t sv[2] = { best & 0xffffu, best >> 16 };
#pragma unroll
                for( int h = 0; h < 2; h++ ) {
                    if( slots[h] == 0xffffffffu )
                        continue;
                    int32_t * dst = p.sink.score + (uint64_t) slots[h] * p.sink.score_stride + id;
                    if( cross[h] == INT_MAX ) {
                        *dst = (int32_t) (sv[h] - QP_BIAS);
                    }
                    else {
                        *dst = 255;
                        unsigned q = atomicAdd( p.sink.next_count, 1u );
                        if( q < p.sink.next_cap )
                            p.sink.next[q] = PairTask{ slots[h], id, cross[h] + 1, 0 };
                        else
                            atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                    }
                }
            }
        }
    }
}

// grid == 0: report the resident CTAs per SM in *blocks_per_sm without launching.
template <int R, int MB, bool HM, int G = QP_G>
static cudaError_t launch_qp4_one( const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    const size_t smem = (size_t) (QP_THREADS / 32) * QP_CODES * G * R * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute( sw_qpair4_kernel<R, MB, HM, G>,
            cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, sw_qpair4_kernel<R, MB, HM, G>,
                QP_THREADS, smem );
    sw_qpair4_kernel<R, MB, HM, G><<<grid, QP_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

// hmax: the running maximum in fp16x2 (4 resident CTAs per SM only);
// g8: the class of 96 rows per pass (R = 24) as 8 threads of 12 rows
cudaError_t launch_sw_qpair4( int R, int mb, bool hmax, bool g8, const QPairParams & p, int grid, cudaStream_t st,
        int * blocks_per_sm ) {
    if( g8 ) {
        if( R != 24 || hmax )
            return cudaErrorInvalidValue;
        return mb == 5 ? launch_qp4_one<12, 5, false, 8>( p, grid, st, blocks_per_sm )
                       : launch_qp4_one<12, 4, false, 8>( p, grid, st, blocks_per_sm );
    }
#define SSA_QP4_CASE( RR ) \
    case RR: \
        return hmax ? launch_qp4_one<RR, 4, true>( p, grid, st, blocks_per_sm ) \
                    : mb == 5 ? launch_qp4_one<RR, 5, false>( p, grid, st, blocks_per_sm ) \
                              : launch_qp4_one<RR, 4, false>( p, grid, st, blocks_per_sm );
    switch( R ) {
    SSA_QP4_CASE( 16 )
    SSA_QP4_CASE( 20 )
    SSA_QP4_CASE( 24 )
    SSA_QP4_CASE( 28 )
    default:
        return cudaErrorInvalidValue;
    }
#undef SSA_QP4_CASE
}

// grid == 0: report the resident CTAs per SM in *blocks_per_sm without launching.
template <int R, int MB>
static cudaError_t launch_qp_one( const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    const size_t smem = (size_t) (QP_THREADS / 32) * QP_CODES * QP_G * R * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute( sw_qpair_kernel<R, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, sw_qpair_kernel<R, MB>, QP_THREADS,
                smem );
    sw_qpair_kernel<R, MB><<<grid, QP_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_sw_qpair( int R, int mb, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
#define SSA_QP_CASE( RR ) \
    case RR: \
        return mb == 5 ? launch_qp_one<RR, 5>( p, grid, st, blocks_per_sm ) \
                       : launch_qp_one<RR, 4>( p, grid, st, blocks_per_sm );
    switch( R ) {
    SSA_QP_CASE( 16 )
    SSA_QP_CASE( 20 )
    SSA_QP_CASE( 24 )
    SSA_QP_CASE( 28 )
    default:
        return cudaErrorInvalidValue;
    }
#undef SSA_QP_CASE
}

// ---------------------------------------------------------------------------
// Needleman-Wunsch, 16-bit entry (reference: src/algo/simd/search_simd_nw.c:
// 180-516, boundaries :233-240, :445-453; the score is H of the last query
// row at the sequence's last column).  The reference lane computes saturating
// int16 values and re-queues the sequence when a block's minimum comes near
// -32768 or its maximum reaches 32767.  The host passes, per query pair, the
// longest sequence for which every value of the matrix (padded rows and the
// last block's pad columns included) provably stays within +-30000: for those
// the lane never saturates and never re-queues, so exact arithmetic gives its
// score.  Longer sequences go to a list that the lane emulation runs.
//
// Values carry a +32768 bias per half and use unsigned 16x2 arithmetic, so
// adding the 32-bit constant gapO + gapE to a word carries exactly once out of
// the low half.  Same wavefront, two interleaved columns per step and profile
// slices as sw_qpair_kernel; there is no zero floor and no running maximum.
// ---------------------------------------------------------------------------
constexpr uint32_t NWQ_BIAS = 32768u;

__device__ __forceinline__ uint32_t nw_pack( int32_t v ) {
    const uint32_t u = (uint32_t) (v + (int32_t) NWQ_BIAS) & 0xffffu;
    return u | (u << 16);
}

// one step's rows: column c (cell A, row r) interleaved with column c + 1
// (cell B, row r - 1); CAPTURE records H at the queries' last rows when one
// of the two columns is the sequence's last
template <int R, bool CAPTURE>
__device__ __forceinline__ void nw_rows( uint32_t (&H)[R], uint32_t (&E)[R], const uint32_t * pa,
        const uint32_t * pb, uint32_t diag, uint32_t up_h0, uint32_t & fa, uint32_t & fb, uint32_t GOE32,
        uint32_t GE2, int32_t row0, bool last_a, bool last_b, int32_t qa_last, int32_t qb_last, uint32_t & cap_a,
        uint32_t & cap_b, uint32_t & out_h0 ) {
    uint4 xa = make_uint4( 0, 0, 0, 0 ), xb = xa;
    uint32_t hc_prev = 0, hc_prev2 = 0;
#pragma unroll
    for( int r = 0; r <= R; r++ ) {
        uint32_t ha = 0;
        if( r < R ) {
            if( (r & 3) == 0 )
                xa = *reinterpret_cast<const uint4 *>( pa + r );
            const uint32_t v = (r & 3) == 0 ? xa.x : (r & 3) == 1 ? xa.y : (r & 3) == 2 ? xa.z : xa.w;
            const uint32_t hd = (r == 0) ? diag : H[r - 1];
            ha = __viaddmax_u16x2( hd, v, __vmaxu2( E[r], fa ) );
            const uint32_t hg = ha + GOE32;
            fa = __viaddmax_u16x2( fa, GE2, hg );
            E[r] = __viaddmax_u16x2( E[r], GE2, hg );
            if constexpr( CAPTURE ) {
                if( last_a && row0 + r == qa_last )
                    cap_a = ha;
                if( last_a && row0 + r == qb_last )
                    cap_b = ha;
            }
        }
        if( r >= 1 ) {
            const int rb = r - 1;
            if( (rb & 3) == 0 )
                xb = *reinterpret_cast<const uint4 *>( pb + rb );
            const uint32_t v = (rb & 3) == 0 ? xb.x : (rb & 3) == 1 ? xb.y : (rb & 3) == 2 ? xb.z : xb.w;
            const uint32_t hd = (rb == 0) ? up_h0 : hc_prev2;
            const uint32_t hb = __viaddmax_u16x2( hd, v, __vmaxu2( E[rb], fb ) );
            const uint32_t hg = hb + GOE32;
            fb = __viaddmax_u16x2( fb, GE2, hg );
            E[rb] = __viaddmax_u16x2( E[rb], GE2, hg );
            H[rb] = hb;
            if constexpr( CAPTURE ) {
                if( last_b && row0 + rb == qa_last )
                    cap_a = hb;
                if( last_b && row0 + rb == qb_last )
                    cap_b = hb;
            }
        }
        hc_prev2 = hc_prev;
        hc_prev = ha;
    }
    out_h0 = hc_prev2;
}

template <int R>
__global__ void __launch_bounds__( QP_THREADS, 4 ) nw_qpair_kernel( QPairParams p ) {
    constexpr int G = QP_G;
    constexpr uint32_t GR = (uint32_t) (G * R);
    extern __shared__ __align__( 16 ) uint32_t qsm[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t * slice = qsm + warp_in_cta * (QP_CODES * GR);
    const int k = lane & (G - 1);
    const int g = lane / G;
    const int gO = p.gap_open, gE = p.gap_e;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) gE << 16) | (uint16_t) (int16_t) gE;
    int4 * scratch = p.scratch + ((uint64_t) warp_global * QP_GPW + (uint32_t) g) * p.scratch_cols;
    uint64_t loaded_key = ~0ull;
    // exact NW boundaries (no saturation within the guarded range)
    auto left_h = [&]( int32_t i ) { return gO + (i + 1) * gE; };           // H(i, -1)
    auto left_e = [&]( int32_t i ) { return 2 * gO + (i + 2) * gE; };       // E entering column 0
    auto top_h = [&]( int32_t j ) { return j < 0 ? 0 : gO + (j + 1) * gE; };   // H(-1, j)
    auto top_f = [&]( int32_t c ) { return 2 * gO + (c + 2) * gE; };        // F entering row 0

    for( ;; ) {
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t qp = p.unit_pairs[u / p.n_chunks];
        const uint32_t chunk = (uint32_t) (u % p.n_chunks);
        const uint32_t seq_begin = p.chunk_bounds[chunk], seq_end = p.chunk_bounds[chunk + 1];
        const uint32_t rows = p.qp_rows[qp];
        const uint32_t passes = rows / GR;
        const uint32_t * prof = p.prof + p.prof_off[qp];
        const uint32_t slot_a = p.qp_slots[2 * qp], slot_b = p.qp_slots[2 * qp + 1];
        const int32_t qa_last = (int32_t) p.qlen[slot_a] - 1;
        const int32_t qb_last = (slot_b == 0xffffffffu) ? -1 : (int32_t) p.qlen[slot_b] - 1;
        const uint32_t lmax = p.qp_lmax[qp];

        for( uint32_t b0 = seq_begin; b0 < seq_end; b0 += (uint32_t) QP_GPW ) {
            const uint32_t idx = b0 + (uint32_t) g;
            const bool valid = idx < seq_end;
            const uint32_t id = valid ? p.order[idx] : 0u;
            const uint32_t L = valid ? p.db.lens[id] : 0u;
            const bool exact = valid && L <= lmax;
            if( valid && !exact && k == 0 ) {
                // beyond the guarded range: the lane emulation scores it
                const uint32_t slots[2] = { slot_a, slot_b };
                for( int h = 0; h < 2; h++ ) {
                    if( slots[h] == 0xffffffffu )
                        continue;
                    const unsigned q = atomicAdd( p.redo_count, 1u );
                    if( q < p.redo_cap )
                        p.redo[q] = PairTask{ slots[h], id, 0, 0 };
                    else
                        atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                }
            }
            const uint32_t ncp = exact ? (((L + 3u) & ~3u) >> 1) : 0u;
            const uint32_t max_ncp = __reduce_max_sync( 0xffffffffu, ncp );
            if( max_ncp == 0 )
                continue;
            const uint8_t * res = p.db.codes + (valid ? p.db.offsets[id] : 0ull);
            const int32_t last_col = (int32_t) L - 1;
            const int32_t cap_cp = last_col >> 1;
            const bool last_is_a = (last_col & 1) == 0;
            uint32_t cap_a = 0, cap_b = 0;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool last_pass = (pass + 1 == passes);
                const uint64_t key = ((uint64_t) qp << 24) | pass;
                if( key != loaded_key ) {
                    __syncwarp();
                    constexpr uint32_t per_code = GR / 4u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < QP_CODES * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 4u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                const int32_t row0 = (int32_t) (pass * GR) + k * R;
                // does this thread hold a query's last row in this pass?
                const bool holds_last = (qa_last >= row0 && qa_last < row0 + R) ||
                        (qb_last >= row0 && qb_last < row0 + R);
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = nw_pack( left_h( row0 + r ) );
                    E[r] = nw_pack( left_e( row0 + r ) );
                }
                uint32_t diag = nw_pack( row0 == 0 ? 0 : left_h( row0 - 1 ) );
                uint32_t out_h0 = 0, out_f0 = 0, out_h1 = 0, out_f1 = 0;
                const uint32_t fetch_limit = ncp + 3u;
                auto fetch = [&]( int32_t cp ) -> uint32_t {
                    const uint32_t c = min( (uint32_t) max( cp, 0 ), fetch_limit );
                    return (uint32_t) *reinterpret_cast<const uint16_t *>( res + 2u * c );
                };
                uint32_t q0 = fetch( -k ), q1 = fetch( 1 - k ), q2 = fetch( 2 - k ), q3 = fetch( 3 - k );
                const bool reads_boundary = (k == 0) && pass > 0;
                int4 bq0 = make_int4( 0, 0, 0, 0 ), bq1 = bq0;
                if( reads_boundary ) {
                    if( ncp > 0 )
                        bq0 = scratch[0];
                    if( ncp > 1 )
                        bq1 = scratch[1];
                }
                const uint32_t steps = max_ncp + (uint32_t) G - 1u;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h0 = __shfl_up_sync( 0xffffffffu, out_h0, 1, G );
                    uint32_t up_f0 = __shfl_up_sync( 0xffffffffu, out_f0, 1, G );
                    uint32_t up_h1 = __shfl_up_sync( 0xffffffffu, out_h1, 1, G );
                    uint32_t up_f1 = __shfl_up_sync( 0xffffffffu, out_f1, 1, G );
                    const int32_t cp = (int32_t) s - k;
                    const uint32_t w = q0;
                    q0 = q1;
                    q1 = q2;
                    q2 = q3;
                    q3 = fetch( cp + 4 );
                    const int4 bnd = bq0;
                    if( reads_boundary ) {
                        bq0 = bq1;
                        const uint32_t nxt = (uint32_t) cp + 2u;
                        if( nxt < ncp && nxt < p.scratch_cols )
                            bq1 = scratch[nxt];
                    }
                    if( cp < 0 || (uint32_t) cp >= ncp )
                        continue;
                    if( k == 0 ) {
                        if( pass ) {
                            up_h0 = (uint32_t) bnd.x;
                            up_f0 = (uint32_t) bnd.y;
                            up_h1 = (uint32_t) bnd.z;
                            up_f1 = (uint32_t) bnd.w;
                        }
                        else {
                            const int32_t c = 2 * cp;
                            up_h0 = nw_pack( top_h( c ) );
                            up_f0 = nw_pack( top_f( c ) );
                            up_h1 = nw_pack( top_h( c + 1 ) );
                            up_f1 = nw_pack( top_f( c + 1 ) );
                        }
                    }
                    const uint32_t * pa = slice + (w & 0xffu) * GR + (uint32_t) (k * R);
                    const uint32_t * pb = slice + (w >> 8) * GR + (uint32_t) (k * R);
                    uint32_t fa = up_f0, fb = up_f1;
                    if( holds_last && cp == cap_cp )
                        nw_rows<R, true>( H, E, pa, pb, diag, up_h0, fa, fb, GOE32, GE2, row0, last_is_a, !last_is_a,
                                qa_last, qb_last, cap_a, cap_b, out_h0 );
                    else
                        nw_rows<R, false>( H, E, pa, pb, diag, up_h0, fa, fb, GOE32, GE2, row0, false, false,
                                qa_last, qb_last, cap_a, cap_b, out_h0 );
                    diag = up_h1;
                    out_f0 = fa;
                    out_h1 = H[R - 1];
                    out_f1 = fb;
                    if( k == G - 1 && !last_pass ) {
                        if( (uint32_t) cp < p.scratch_cols )
                            scratch[cp] = make_int4( (int) out_h0, (int) out_f0, (int) out_h1, (int) out_f1 );
                        else
                            atomicOr( p.sink.error_flags, ERR_SCRATCH_OVERFLOW );
                    }
                }
                __syncwarp();
            }
            // the threads holding the last rows report (values are > 0 with the bias)
#pragma unroll
            for( int o = 1; o < G; o <<= 1 ) {
                cap_a = max( cap_a, __shfl_xor_sync( 0xffffffffu, cap_a, o, G ) );
                cap_b = max( cap_b, __shfl_xor_sync( 0xffffffffu, cap_b, o, G ) );
            }
            if( exact && k == 0 ) {
                p.sink.score[(uint64_t) slot_a * p.sink.score_stride + id] =
                        (int32_t) (cap_a & 0xffffu) - (int32_t) NWQ_BIAS;
                if( slot_b != 0xffffffffu )
                    p.sink.score[(uint64_t) slot_b * p.sink.score_stride + id] =
                            (int32_t) (cap_b >> 16) - (int32_t) NWQ_BIAS;
            }
        }
    }
}

template <int R>
static cudaError_t launch_nw_one( const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    const size_t smem = (size_t) (QP_THREADS / 32) * QP_CODES * QP_G * R * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute( nw_qpair_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, nw_qpair_kernel<R>, QP_THREADS, smem );
    nw_qpair_kernel<R><<<grid, QP_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_nw_qpair( int R, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    switch( R ) {
    case 16:
        return launch_nw_one<16>( p, grid, st, blocks_per_sm );
    case 20:
        return launch_nw_one<20>( p, grid, st, blocks_per_sm );
    case 24:
        return launch_nw_one<24>( p, grid, st, blocks_per_sm );
    case 28:
        return launch_nw_one<28>( p, grid, st, blocks_per_sm );
    default:
        return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Needleman-Wunsch, 16-bit entry, one 4-column block per step.  Arithmetic,
// boundaries, exact range and redo list are those of nw_qpair_kernel; the
// block layout is that of sw_qpair4_kernel: chain j of a thread computes
// column 4b + j, the four chains run skewed by one row (iteration it holds
// cell (it - j, 4b + j) of every chain), a 4-byte load brings a block's
// residues, and a pass boundary carries H and F of the four columns in two
// int4.  A query's score is H at its last row in the sequence's last column
// L - 1, i.e. block (L - 1) / 4, chain (L - 1) % 4.
// ---------------------------------------------------------------------------

// One block of R rows and four columns.  up_h[j]: H of the row above this
// thread's first row in column 4b + j; f[j]: F entering the first row (on
// return: F leaving the last row); out_h[j]: H of the last row.  CAPTURE:
// record chain jl's H at rows ra and rb (a query's last row, relative to
// the thread's first row) in cap_a / cap_b.
template <int R, bool CAPTURE>
__device__ __forceinline__ void nw4_block( uint32_t (&H)[R], uint32_t (&E)[R], const uint32_t * const (&pc)[4],
        uint32_t diag, const uint32_t (&up_h)[4], uint32_t (&f)[4], uint32_t (&out_h)[4], uint32_t GOE32,
        uint32_t GE2, int jl, int ra, int rb, uint32_t & cap_a, uint32_t & cap_b ) {
    constexpr int C = 4;
    uint4 x[C];
    // hv[j][r]: H of chain j at row r; only the last two rows of chains 0..2
    // stay live
    uint32_t hv[C][R];
#pragma unroll
    for( int it = 0; it < R + C - 1; it++ ) {
#pragma unroll
        for( int j = 0; j < C; j++ ) {
            const int r = it - j;
            if( r < 0 || r >= R )
                continue;
            if( (r & 3) == 0 )
                x[j] = *reinterpret_cast<const uint4 *>( pc[j] + r );
            const uint32_t v = (r & 3) == 0 ? x[j].x : (r & 3) == 1 ? x[j].y : (r & 3) == 2 ? x[j].z : x[j].w;
            uint32_t hd;
            if( r == 0 )
                hd = (j == 0) ? diag : up_h[j - 1];
            else
                hd = (j == 0) ? H[r - 1] : hv[j - 1][r - 1];
            const uint32_t h = __viaddmax_u16x2( hd, v, __vmaxu2( E[r], f[j] ) );
            const uint32_t hg = h + GOE32;
            f[j] = __viaddmax_u16x2( f[j], GE2, hg );
            E[r] = __viaddmax_u16x2( E[r], GE2, hg );
            hv[j][r] = h;
            if constexpr( CAPTURE ) {
                if( j == jl && r == ra )
                    cap_a = h;
                if( j == jl && r == rb )
                    cap_b = h;
            }
            // chain 3 leaves column 4b + 3 in H (chain 0 of this block has
            // read H[r] at iteration r + 1 < r + 3)
            if( j == C - 1 )
                H[r] = h;
        }
    }
#pragma unroll
    for( int j = 0; j < C; j++ )
        out_h[j] = hv[j][R - 1];
}

// Pass-boundary staging of nw_qpair4_kernel: thread 0 of a group copies the
// boundary row of block b + NW4_AHEAD into a ring of NW4_SLOTS shared-memory
// slots (two int4 each) with cp.async while it computes block b, instead of
// holding the prefetched row in registers.  One commit group per block (empty
// past the last block), so waiting until at most NW4_AHEAD - 1 groups are in
// flight leaves block b's copy complete.  The slot written at step b is the
// one read at step b - 1, whose values that step has already consumed.
constexpr int NW4_AHEAD = 2;
constexpr int NW4_SLOTS = NW4_AHEAD + 1;

__device__ __forceinline__ void cp_async16( void * smem, const void * gmem ) {
    const uint32_t s = (uint32_t) __cvta_generic_to_shared( smem );
    asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;" ::"r"( s ), "l"( gmem ) : "memory" );
}

__device__ __forceinline__ void cp_async_commit() {
    asm volatile( "cp.async.commit_group;" ::: "memory" );
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile( "cp.async.wait_group %0;" ::"n"( N ) : "memory" );
}

// shared memory of nw_qpair4_kernel: the warps' profile slices, then the
// groups' boundary rings
template <int R>
constexpr size_t nw4_smem_bytes() {
    return (size_t) (QP_THREADS / 32) * QP_CODES * QP_G * R * sizeof(uint32_t) +
            (size_t) (QP_THREADS / QP_G) * NW4_SLOTS * 2 * sizeof(int4);
}

template <int R>
__global__ void __launch_bounds__( QP_THREADS, 4 ) nw_qpair4_kernel( QPairParams p ) {
    constexpr int G = QP_G;
    constexpr int C = 4;
    constexpr uint32_t GR = (uint32_t) (G * R);
    extern __shared__ __align__( 16 ) uint32_t qsm[];
    const int lane = threadIdx.x & 31;
    const uint32_t warp_in_cta = threadIdx.x >> 5;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t * slice = qsm + warp_in_cta * (QP_CODES * GR);
    const int k = lane & (G - 1);
    const int g = lane / G;
    const int gO = p.gap_open, gE = p.gap_e;
    const uint32_t GOE32 = (uint32_t) ((int32_t) p.gap_oe * 65536 + (int32_t) p.gap_oe);
    const uint32_t GE2 = ((uint32_t) (uint16_t) (int16_t) gE << 16) | (uint16_t) (int16_t) gE;
    int4 * scratch = p.scratch + ((uint64_t) warp_global * QP_GPW + (uint32_t) g) * p.scratch_cols;
    // this group's boundary ring, after all warps' profile slices
    int4 * ring = reinterpret_cast<int4 *>( qsm + (QP_THREADS / 32) * (QP_CODES * GR) ) +
            (size_t) (threadIdx.x / G) * (NW4_SLOTS * 2);
    uint64_t loaded_key = ~0ull;
    auto left_h = [&]( int32_t i ) { return gO + (i + 1) * gE; };           // H(i, -1)
    auto left_e = [&]( int32_t i ) { return 2 * gO + (i + 2) * gE; };       // E entering column 0
    auto top_h = [&]( int32_t j ) { return j < 0 ? 0 : gO + (j + 1) * gE; };   // H(-1, j)
    auto top_f = [&]( int32_t c ) { return 2 * gO + (c + 2) * gE; };        // F entering row 0

    for( ;; ) {
        unsigned long long u = 0;
        if( lane == 0 )
            u = atomicAdd( p.unit_counter, 1ull );
        u = __shfl_sync( 0xffffffffu, u, 0 );
        if( u >= p.n_units )
            break;
        const uint32_t qp = p.unit_pairs[u / p.n_chunks];
        const uint32_t chunk = (uint32_t) (u % p.n_chunks);
        const uint32_t seq_begin = p.chunk_bounds[chunk], seq_end = p.chunk_bounds[chunk + 1];
        const uint32_t rows = p.qp_rows[qp];
        const uint32_t passes = rows / GR;
        const uint32_t * prof = p.prof + p.prof_off[qp];
        const uint32_t slot_a = p.qp_slots[2 * qp], slot_b = p.qp_slots[2 * qp + 1];
        const int32_t qa_last = (int32_t) p.qlen[slot_a] - 1;
        const int32_t qb_last = (slot_b == 0xffffffffu) ? -1 : (int32_t) p.qlen[slot_b] - 1;
        const uint32_t lmax = p.qp_lmax[qp];

        for( uint32_t b0 = seq_begin; b0 < seq_end; b0 += (uint32_t) QP_GPW ) {
            const uint32_t idx = b0 + (uint32_t) g;
            const bool valid = idx < seq_end;
            const uint32_t id = valid ? p.order[idx] : 0u;
            const uint32_t L = valid ? p.db.lens[id] : 0u;
            const bool exact = valid && L <= lmax;
            if( valid && !exact && k == 0 ) {
                // beyond the guarded range: the lane emulation scores it
                const uint32_t slots[2] = { slot_a, slot_b };
                for( int h = 0; h < 2; h++ ) {
                    if( slots[h] == 0xffffffffu )
                        continue;
                    const unsigned q = atomicAdd( p.redo_count, 1u );
                    if( q < p.redo_cap )
                        p.redo[q] = PairTask{ slots[h], id, 0, 0 };
                    else
                        atomicOr( p.sink.error_flags, ERR_REQUEUE_OVERFLOW );
                }
            }
            const uint32_t nb = exact ? (L + 3u) >> 2 : 0u;         // 4-column blocks
            const uint32_t max_nb = __reduce_max_sync( 0xffffffffu, nb );
            if( max_nb == 0 )
                continue;
            const uint8_t * res = p.db.codes + (valid ? p.db.offsets[id] : 0ull);
            const int32_t last_col = (int32_t) L - 1;
            const int32_t cap_blk = last_col >> 2;
            const int jl = last_col & 3;
            uint32_t cap_a = 0, cap_b = 0;

            for( uint32_t pass = 0; pass < passes; pass++ ) {
                const bool last_pass = (pass + 1 == passes);
                const uint64_t key = ((uint64_t) qp << 24) | pass;
                if( key != loaded_key ) {
                    __syncwarp();
                    constexpr uint32_t per_code = GR / 4u;
                    const uint4 * src = reinterpret_cast<const uint4 *>( prof + (size_t) pass * GR );
                    uint4 * dst = reinterpret_cast<uint4 *>( slice );
                    for( uint32_t i = (uint32_t) lane; i < QP_CODES * per_code; i += 32u ) {
                        const uint32_t code = i / per_code, w = i % per_code;
                        dst[i] = src[(size_t) code * (rows / 4u) + w];
                    }
                    loaded_key = key;
                    __syncwarp();
                }
                const int32_t row0 = (int32_t) (pass * GR) + k * R;
                const int ra = qa_last - row0, rb = qb_last - row0;
                // does this thread hold a query's last row in this pass?
                const bool holds_last = (ra >= 0 && ra < R) || (rb >= 0 && rb < R);
                uint32_t H[R], E[R];
#pragma unroll
                for( int r = 0; r < R; r++ ) {
                    H[r] = nw_pack( left_h( row0 + r ) );
                    E[r] = nw_pack( left_e( row0 + r ) );
                }
                uint32_t diag = nw_pack( row0 == 0 ? 0 : left_h( row0 - 1 ) );
                uint32_t out_h[C], out_f[C];
#pragma unroll
                for( int j = 0; j < C; j++ ) {
                    out_h[j] = 0;
                    out_f[j] = 0;
                }
                // residues of blocks b and b + 1, one block fetched two steps
                // ahead (a step takes thousands of cycles); past the last block
                // the reads stay inside the padded record or the next one
                // (never used)
                const uint32_t fetch_limit = nb + 3u;
                auto fetch = [&]( int32_t b ) -> uint32_t {
                    const uint32_t c = min( (uint32_t) max( b, 0 ), fetch_limit );
                    return __ldcs( reinterpret_cast<const unsigned int *>( res + 4u * c ) );
                };
                uint32_t q0 = fetch( -k ), q1 = fetch( 1 - k );
                // thread 0: the previous pass's bottom row, NW4_AHEAD blocks
                // ahead through the ring
                const bool reads_boundary = (k == 0) && pass > 0;
                if( reads_boundary ) {
#pragma unroll
                    for( int x = 0; x < NW4_AHEAD; x++ ) {
                        if( (uint32_t) x < nb && 2u * (uint32_t) x + 1u < p.scratch_cols ) {
                            cp_async16( ring + 2 * x, scratch + 2 * x );
                            cp_async16( ring + 2 * x + 1, scratch + 2 * x + 1 );
                        }
                        cp_async_commit();
                    }
                }
                const uint32_t steps = max_nb + (uint32_t) G - 1u;
                for( uint32_t s = 0; s < steps; s++ ) {
                    uint32_t up_h[C], up_f[C];
#pragma unroll
                    for( int j = 0; j < C; j++ ) {
                        up_h[j] = __shfl_up_sync( 0xffffffffu, out_h[j], 1, G );
                        up_f[j] = __shfl_up_sync( 0xffffffffu, out_f[j], 1, G );
                    }
                    const int32_t b = (int32_t) s - k;
                    const uint32_t w = q0;
                    q0 = q1;
                    q1 = fetch( b + 2 );
                    if( b < 0 || (uint32_t) b >= nb )
                        continue;
                    if( k == 0 ) {
                        if( pass ) {
                            // block b's copy is complete once at most
                            // NW4_AHEAD - 1 later groups are in flight
                            cp_async_wait<NW4_AHEAD - 1>();
                            const uint32_t slot = (uint32_t) b % (uint32_t) NW4_SLOTS;
                            const int4 bnd0 = ring[2 * slot], bnd1 = ring[2 * slot + 1];
                            const uint32_t nxt = (uint32_t) b + (uint32_t) NW4_AHEAD;
                            if( nxt < nb && 2u * nxt + 1u < p.scratch_cols ) {
                                const uint32_t ns = nxt % (uint32_t) NW4_SLOTS;
                                cp_async16( ring + 2 * ns, scratch + 2u * nxt );
                                cp_async16( ring + 2 * ns + 1, scratch + 2u * nxt + 1u );
                            }
                            cp_async_commit();
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
                            const int32_t c = 4 * b;
#pragma unroll
                            for( int j = 0; j < C; j++ ) {
                                up_h[j] = nw_pack( top_h( c + j ) );
                                up_f[j] = nw_pack( top_f( c + j ) );
                            }
                        }
                    }
                    const uint32_t * pc[C];
#pragma unroll
                    for( int j = 0; j < C; j++ )
                        pc[j] = slice + ((w >> (8 * j)) & 0xffu) * GR + (uint32_t) (k * R);
                    uint32_t f[C];
#pragma unroll
                    for( int j = 0; j < C; j++ )
                        f[j] = up_f[j];
                    if( holds_last && b == cap_blk )
                        nw4_block<R, true>( H, E, pc, diag, up_h, f, out_h, GOE32, GE2, jl, ra, rb, cap_a, cap_b );
                    else
                        nw4_block<R, false>( H, E, pc, diag, up_h, f, out_h, GOE32, GE2, jl, ra, rb, cap_a, cap_b );
                    diag = up_h[C - 1];
#pragma unroll
                    for( int j = 0; j < C; j++ )
                        out_f[j] = f[j];
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
                // every copy issued was for a block this pass computed and
                // waited for; drain the (empty) groups before the ring's reuse
                if( reads_boundary )
                    cp_async_wait<0>();
                __syncwarp();
            }
            // the threads holding the last rows report (values are > 0 with the bias)
#pragma unroll
            for( int o = 1; o < G; o <<= 1 ) {
                cap_a = max( cap_a, __shfl_xor_sync( 0xffffffffu, cap_a, o, G ) );
                cap_b = max( cap_b, __shfl_xor_sync( 0xffffffffu, cap_b, o, G ) );
            }
            if( exact && k == 0 ) {
                p.sink.score[(uint64_t) slot_a * p.sink.score_stride + id] =
                        (int32_t) (cap_a & 0xffffu) - (int32_t) NWQ_BIAS;
                if( slot_b != 0xffffffffu )
                    p.sink.score[(uint64_t) slot_b * p.sink.score_stride + id] =
                            (int32_t) (cap_b >> 16) - (int32_t) NWQ_BIAS;
            }
        }
    }
}

template <int R>
static cudaError_t launch_nw4_one( const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    const size_t smem = nw4_smem_bytes<R>();
    cudaError_t e = cudaFuncSetAttribute( nw_qpair4_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) smem );
    if( e != cudaSuccess )
        return e;
    if( grid == 0 )
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor( blocks_per_sm, nw_qpair4_kernel<R>, QP_THREADS, smem );
    nw_qpair4_kernel<R><<<grid, QP_THREADS, smem, st>>>( p );
    return cudaGetLastError();
}

cudaError_t launch_nw_qpair4( int R, const QPairParams & p, int grid, cudaStream_t st, int * blocks_per_sm ) {
    switch( R ) {
    case 16:
        return launch_nw4_one<16>( p, grid, st, blocks_per_sm );
    case 20:
        return launch_nw4_one<20>( p, grid, st, blocks_per_sm );
    case 24:
        return launch_nw4_one<24>( p, grid, st, blocks_per_sm );
    case 28:
        return launch_nw4_one<28>( p, grid, st, blocks_per_sm );
    default:
        return cudaErrorInvalidValue;
    }
}

// prof[qp][code][row] = (A's score, B's score) as a 16x2 word at the entry
// width; rows past a query, and the absent query of an odd batch, score -128
// (8-bit Smith-Waterman: never raises a maximum) or 0 (16-bit
// Needleman-Wunsch: rows below a query do not feed back into it).
__global__ void build_profile_qp_kernel( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qp_slots, uint32_t n_qp, const uint32_t * qp_rows, const int64_t * matrix, uint32_t * prof,
        const uint64_t * prof_off, int width ) {
    const uint32_t qp = blockIdx.y;
    if( qp >= n_qp )
        return;
    const uint32_t rows = qp_rows[qp];
    const uint32_t sa = qp_slots[2 * qp], sb = qp_slots[2 * qp + 1];
    const uint32_t La = qlen[sa], Lb = (sb == 0xffffffffu) ? 0u : qlen[sb];
    const uint8_t * qa = qcodes + qoff[sa];
    const uint8_t * qb = (sb == 0xffffffffu) ? qa : qcodes + qoff[sb];
    uint32_t * out = prof + prof_off[qp];
    for( uint64_t x = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; x < (uint64_t) QP_CODES * rows;
            x += (uint64_t) gridDim.x * blockDim.x ) {
        const uint32_t code = (uint32_t) (x / rows), row = (uint32_t) (x % rows);
        const int32_t pad = (width == 8) ? -128 : 0;
        int32_t a = pad, b = pad;
        if( row < La ) {
            const int64_t m = matrix[(code << 5) + qa[row]];
            a = (width == 8) ? (int32_t) (int8_t) m : (int32_t) (int16_t) m;
        }
        if( row < Lb ) {
            const int64_t m = matrix[(code << 5) + qb[row]];
            b = (width == 8) ? (int32_t) (int8_t) m : (int32_t) (int16_t) m;
        }
        out[x] = ((uint32_t) (uint16_t) (int16_t) b << 16) | (uint16_t) (int16_t) a;
    }
}

cudaError_t launch_build_profile_qp( const uint8_t * qcodes, const uint64_t * qoff, const uint32_t * qlen,
        const uint32_t * qp_slots, uint32_t n_qp, const uint32_t * qp_rows, const int64_t * matrix, uint32_t * prof,
        const uint64_t * prof_off, int width, cudaStream_t st ) {
    if( n_qp == 0 )
        return cudaSuccess;
    dim3 grid( 16, n_qp );
    build_profile_qp_kernel<<<grid, 256, 0, st>>>( qcodes, qoff, qlen, qp_slots, n_qp, qp_rows, matrix, prof,
            prof_off, width );
    return cudaGetLastError();
}

}  // namespace ssa
