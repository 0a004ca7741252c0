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
// Each pass is a warp wavefront: lane k owns query rows [stripe*256 + 8k, +8),
// database columns stream through the warp, the bottom row of a lane goes to
// the next lane by shuffle.  A hit runs on a group of 1 or 4 warps
// (stripe_pipeline.cuh): stripe i on warp i % W, its bottom row handed to the
// next stripe through shared memory or the group's boundary row in global
// memory.  All arithmetic is exact (int32, with the host guaranteeing the
// range), matching the reference's int64 code.
#include "device_common.cuh"
#include "stripe_pipeline.cuh"

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


// Per-hit setup shared by the passes: the group's warps, its shared state and
// boundary row in global memory (stripe_pipeline.cuh).
template <int W>
struct TbGroup {
    static constexpr int GROUPS = 256 / (32 * W);
    int lane, wig, g;
    PipeShared<W> * sh;
    GroupBarrier<W> gb;
    int4 * scratch;
    uint32_t scratch_cols;
    __device__ TbGroup( PipeShared<W> * shs, const TbParams & p ) {
        lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        g = warp / W;
        wig = warp % W;
        sh = &shs[g];
        gb = GroupBarrier<W>{ 1u + (uint32_t) g };
        const uint64_t group = (uint64_t) blockIdx.x * GROUPS + g;
        scratch = p.scratch ? p.scratch + group * p.scratch_cols : nullptr;
        scratch_cols = p.scratch ? p.scratch_cols : 0;
    }
    // the next hit of the counter, the same on every warp of the group
    __device__ uint32_t take( unsigned long long * counter ) {
        if( wig == 0 && lane == 0 )
            sh->item = (uint32_t) atomicAdd( counter, 1ull );
        gb.sync();
        return sh->item;
    }
    template <class Body>
    __device__ void link( Body & body, const int32_t * smat, const TbParams & p ) {
        body.smat = smat;
        body.lane = lane;
        body.gO = p.gap_open;
        body.gE = p.gap_extend;
        body.gOE = p.gap_open + p.gap_extend;
        body.error_flags = p.error_flags;
        body.link.sh = sh;
        body.link.scratch = scratch;
        body.link.scratch_cols = scratch_cols;
        body.link.wig = wig;
    }
};

// Fields and the row-above / bottom-row plumbing common to the stripe bodies.
template <int W>
struct TbStripeBase {
    const int32_t * smat;
    StripeLink<W> link;
    ResidueRing rr;
    int lane;
    int32_t gO, gE, gOE;
    unsigned * error_flags;
    int qa[TB_R];
    int32_t H[TB_R], E[TB_R];
    int32_t diag, out_h, out_f, row0;
    int nvalid;
    // (H, F) above the lane's first row at column c, given the values of the
    // first stripe's top boundary
    __device__ void above( uint32_t s, int32_t c, int32_t top_h, int32_t top_f, int32_t & up_h, int32_t & up_f ) const {
        if( lane == 0 ) {
            if( link.stripe == 0 ) {
                up_h = top_h;
                up_f = top_f;
            }
            else {
                const int2 v = link.above( s, c );
                up_h = v.x;
                up_f = v.y;
            }
        }
    }
    __device__ void put_bottom( int32_t c ) const {
        if( lane == 31 && !link.put( c, out_h, out_f ) )
            atomicOr( error_flags, ERR_SCRATCH_OVERFLOW );
    }
};

// ---------------------------------------------------------------------------
// 1. SW forward region pass (reference: src/algo/align.c:39-82).  The
//    reference iterates database rows outer and query columns inner, scoring
//    matrix[query][db]; the recurrence is symmetric, so the warp streams the
//    database and keeps the query on lanes.  Key of the end cell: largest
//    value, then smallest database index, then smallest query index.
// ---------------------------------------------------------------------------
template <int W>
struct ForwardStripe : TbStripeBase<W> {
    using B_ = TbStripeBase<W>;
    static constexpr int32_t cand = INT32_MAX;
    const uint8_t * a;
    uint32_t A, B;
    int32_t * lh;
    int32_t * le;
    int32_t pv, pi, pj;                       // this stripe's first maximum
    int32_t best_v, best_i, best_j;           // over the warp's stripes

    __device__ void begin( uint32_t stripe ) {
        this->link.stripe = stripe;
        this->link.last = (stripe + 1) * TB_ROWS >= A;
        this->row0 = (int32_t) (stripe * TB_ROWS) + this->lane * TB_R;
        this->nvalid = max( 0, min( TB_R, (int) A - this->row0 ) );
        load_rows( a, this->row0, 1, this->nvalid, this->qa );
#pragma unroll
        for( int r = 0; r < TB_R; r++ ) {
            this->H[r] = 0;                         // HH[j] = 0
            this->E[r] = this->gO + this->gE;       // max(EE = gapO, HH + gapO) + gapE at row 0
        }
        this->diag = 0;
        this->out_h = 0;
        this->out_f = 0;
        pv = 0;
        pi = INT_MAX;
        pj = INT_MAX;
        this->link.start( B, this->lane );
        this->rr.start( this->lane );
    }

    __device__ bool chunk( uint32_t ck, int32_t ) {
        const uint32_t steps = B + 31, s0 = ck * 32;
        const int lane = this->lane;
        const int32_t gE = this->gE, gOE = this->gOE;
        // one wavefront step; edge: some lane may be on a column outside 0..B-1
        auto column = [&]( const uint32_t s, const bool edge ) {
            int32_t up_h = __shfl_up_sync( 0xffffffffu, this->out_h, 1 );
            int32_t up_f = __shfl_up_sync( 0xffffffffu, this->out_f, 1 );
            const int32_t c = (int32_t) s - lane;
            if( edge && (c < 0 || c >= (int32_t) B) )
                return;
            // f starts at gapO: max(gapO, 0 + gapO) + gapE
            this->above( s, c, 0, this->gO + gE, up_h, up_f );
            int32_t f = up_f, hd = this->diag;
            const int d = this->rr.get( s, lane );
            // branch-free rows: the row-to-row chain is a 3-way max, an add and
            // a fused add-max; a lane visits its cells in (column, row) order,
            // so within a stripe the first maximum wins with a strict compare
            int32_t e_last[TB_R];
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t e_in = this->E[r];
                const int32_t t = max( hd + mget( this->smat, d, this->qa[r] ), 0 );
                const int32_t x = __vimax3_s32( t, f, e_in );
                const bool take = (r < this->nvalid) && x > pv;
                pv = take ? x : pv;
                pi = take ? c : pi;
                pj = take ? this->row0 + r : pj;
                e_last[r] = e_in;
                hd = this->H[r];
                this->H[r] = x;
                const int32_t y = x + gOE;
                f = __viaddmax_s32( f, gE, y );
                this->E[r] = __viaddmax_s32( e_in, gE, y );
            }
            if( c == (int32_t) B - 1 ) {
#pragma unroll
                for( int r = 0; r < TB_R; r++ )
                    if( r < this->nvalid ) {
                        lh[this->row0 + r] = this->H[r];
                        le[this->row0 + r] = e_last[r];
                    }
            }
            this->diag = up_h;
            this->out_h = this->H[TB_R - 1];
            this->out_f = f;
            this->put_bottom( c );
        };
        // the residue ring and the boundary prefetch refill at the first step of a chunk
        this->link.step( B, s0, lane );
        this->rr.step( s0, lane );
        const uint32_t s1 = min( s0 + 32, steps );
        if( s0 >= 31 && s1 <= B ) {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, false );
        }
        else {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, true );
        }
        return s0 + 32 < steps;
    }

    // this stripe's first maximum against the earlier stripes' (value desc,
    // database index asc, query index asc)
    __device__ void end() {
        if( pv > best_v || (pv == best_v && pv > 0 && (pi < best_i || (pi == best_i && pj < best_j))) ) {
            best_v = pv;
            best_i = pi;
            best_j = pj;
        }
    }
};

template <int W>
__global__ void __launch_bounds__( 256 ) tb_forward_kernel( TbParams p ) {
    __shared__ PipeShared<W> shs[TbGroup<W>::GROUPS];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, true );
    TbGroup<W> grp( shs, p );
    for( ;; ) {
        const uint32_t h = grp.take( p.hit_counters + 0 );
        if( h >= p.n_hits )
            break;
        const TbHit hit = p.hits[h];
        if( hit.algo == 0 ) {
            ForwardStripe<W> body;
            grp.link( body, smat, p );
            body.A = p.qlen[hit.qslot];
            body.B = p.db.lens[hit.id];
            body.a = p.qcodes + p.qoff[hit.qslot];
            body.lh = p.last_h + p.last_off[h];
            body.le = p.last_e + p.last_off[h];
            body.best_v = 0;
            body.best_i = INT_MAX;
            body.best_j = INT_MAX;
            body.rr = ResidueRing{ grp.sh->residues[grp.wig], 0, p.db.codes + p.db.offsets[hit.id], (int32_t) body.B,
                                   -1 };
            run_stripes<W>( body, *grp.sh, grp.gb, grp.wig, grp.lane, (body.A + TB_ROWS - 1) / TB_ROWS, body.B,
                    p.error_flags );
            // the best key over the warp, then over the group
            int32_t bv = body.best_v, bi = body.best_i, bj = body.best_j;
            for( int o = 16; o > 0; o >>= 1 ) {
                const int32_t v = __shfl_xor_sync( 0xffffffffu, bv, o );
                const int32_t i = __shfl_xor_sync( 0xffffffffu, bi, o );
                const int32_t j = __shfl_xor_sync( 0xffffffffu, bj, o );
                if( v > bv || (v == bv && (i < bi || (i == bi && j < bj))) ) {
                    bv = v;
                    bi = i;
                    bj = j;
                }
            }
            if( grp.lane == 0 ) {
                grp.sh->red[grp.wig][0] = bv;
                grp.sh->red[grp.wig][1] = bi;
                grp.sh->red[grp.wig][2] = bj;
            }
            grp.gb.sync();
            if( grp.wig == 0 && grp.lane == 0 ) {
                for( int k = 1; k < W; k++ ) {
                    const int32_t v = grp.sh->red[k][0], i = grp.sh->red[k][1], j = grp.sh->red[k][2];
                    if( v > bv || (v == bv && (i < bi || (i == bi && j < bj))) ) {
                        bv = v;
                        bi = i;
                        bj = j;
                    }
                }
                TbRegion rg;
                rg.fwd_score = bv;
                rg.a_end = bj;
                rg.b_end = bi;
                rg.a_begin = 0;
                rg.b_begin = 0;
                rg.status = (bv > 0) ? 0 : 1;
                p.regions[h] = rg;
            }
        }
        // every warp is past this hit's shared state before the next hit
        grp.gb.sync();
    }
}

// ---------------------------------------------------------------------------
// 2. SW reverse pass (reference: src/algo/align.c:84-131).  Both sequences
//    are read backwards from the end cell: row j' = a_end - j, column
//    i' = b_end - i.  The boundary row before column 0 is the reference's
//    work row: -1 for query indices <= b_end, the forward pass's last row
//    above that.  The begin cell is the first cell in (i' asc, j' asc) order
//    whose value reaches the forward score; columns past the first column
//    holding a candidate cannot change it, so that column is the group's
//    limit.
// ---------------------------------------------------------------------------
template <int W>
struct ReverseStripe : TbStripeBase<W> {
    const uint8_t * a;
    uint32_t A, B;
    int32_t score, a_end, b_end;
    const int32_t * lh;
    const int32_t * le;
    int32_t hit_i, hit_j;          // the lane's first (i', j') reaching the score, over its finished stripes
    int32_t s_i, s_j;              // the same in the current stripe
    int32_t cand;                  // the lane's first column so far, read by run_stripes after each chunk

    __device__ void begin( uint32_t stripe ) {
        const int lane = this->lane;
        this->link.stripe = stripe;
        this->link.last = (stripe + 1) * TB_ROWS >= A;
        this->row0 = (int32_t) (stripe * TB_ROWS) + lane * TB_R;
        const int32_t row0 = this->row0;
        this->nvalid = max( 0, min( TB_R, (int) A - row0 ) );
        load_rows( a, (int64_t) a_end - row0, -1, this->nvalid, this->qa );
#pragma unroll
        for( int r = 0; r < TB_R; r++ ) {
            const int32_t j = a_end - (row0 + r);     // query index
            int32_t hh = -1, ee = -1;
            if( r < this->nvalid && j > b_end ) {
                hh = lh[j];
                ee = le[j];
            }
            this->H[r] = hh;                                // HH(b_end + 1, j)
            this->E[r] = max( ee, hh + this->gO ) + this->gE;   // EE(b_end, j)
        }
        // diagonal of the lane's first row at column 0: HH(b_end+1, j+1), or 0
        // for the end cell itself
        const int32_t jprev = a_end - (row0 - 1);
        this->diag = (row0 == 0) ? 0 : ((jprev > b_end) ? lh[jprev] : -1);
        s_i = INT_MAX;
        s_j = INT_MAX;
        this->out_h = 0;
        this->out_f = 0;
        this->link.start( B, lane );
        this->rr.start( lane );
    }

    __device__ bool chunk( uint32_t ck, int32_t lim ) {
        // steps up to the limit column on lane 31
        const uint32_t cols = (lim == INT32_MAX) ? B : min( B, (uint32_t) lim + 1u );
        const uint32_t steps = cols + 31, s0 = ck * 32;
        const int lane = this->lane;
        const int32_t gO = this->gO, gE = this->gE, gOE = this->gOE;
        // one wavefront step; edge: some lane may be on a column outside 0..B-1
        auto column = [&]( const uint32_t s, const bool edge ) {
            int32_t up_h = __shfl_up_sync( 0xffffffffu, this->out_h, 1 );
            int32_t up_f = __shfl_up_sync( 0xffffffffu, this->out_f, 1 );
            const int32_t c = (int32_t) s - lane;
            if( edge && (c < 0 || c >= (int32_t) B) )
                return;
            // h starts at -1 per row; f = max(-1, h + gapO) + gapE
            this->above( s, c, -1, max( -1, -1 + gO ) + gE, up_h, up_f );
            const int d = this->rr.get( s, lane );          // database index b_end - c
            int32_t f = up_f, hd = this->diag;               // stripe 0 lane 0: 0 at c == 0, then -1
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t e_in = this->E[r];
                const int32_t x = __vimax3_s32( hd + mget( this->smat, d, this->qa[r] ), f, e_in );
                // the lane visits a stripe's cells in (column, row) order: its
                // first candidate in the stripe is the stripe's best on the lane
                const bool take = (r < this->nvalid) && x >= score && s_i == INT_MAX;
                s_i = take ? c : s_i;
                s_j = take ? this->row0 + r : s_j;
                hd = this->H[r];
                this->H[r] = x;
                const int32_t y = x + gOE;
                f = __viaddmax_s32( f, gE, y );
                this->E[r] = __viaddmax_s32( e_in, gE, y );
            }
            this->diag = up_h;
            this->out_h = this->H[TB_R - 1];
            this->out_f = f;
            this->put_bottom( c );
        };
        // the residue ring and the boundary prefetch refill at the first step of a chunk
        this->link.step( B, s0, lane );
        this->rr.step( s0, lane );
        const uint32_t s1 = min( s0 + 32, steps );
        if( s0 >= 31 && s1 <= B ) {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, false );
        }
        else {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, true );
        }
        cand = min( hit_i, s_i );
        return s0 + 32 < steps;
    }

    // this stripe's first candidate against the earlier stripes' ((i', j') asc)
    __device__ void end() {
        if( s_i < hit_i || (s_i == hit_i && s_j < hit_j) ) {
            hit_i = s_i;
            hit_j = s_j;
        }
    }
};

template <int W>
__global__ void __launch_bounds__( 256 ) tb_reverse_kernel( TbParams p ) {
    __shared__ PipeShared<W> shs[TbGroup<W>::GROUPS];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, true );
    TbGroup<W> grp( shs, p );
    for( ;; ) {
        const uint32_t h = grp.take( p.hit_counters + 1 );
        if( h >= p.n_hits )
            break;
        const TbHit hit = p.hits[h];
        TbRegion rg = p.regions[h];
        if( hit.algo == 0 && rg.status == 0 ) {
            ReverseStripe<W> body;
            grp.link( body, smat, p );
            body.score = rg.fwd_score;
            body.a_end = rg.a_end;
            body.b_end = rg.b_end;
            body.A = (uint32_t) rg.a_end + 1;     // rows j' = 0..a_end
            body.B = (uint32_t) rg.b_end + 1;     // cols i' = 0..b_end
            body.a = p.qcodes + p.qoff[hit.qslot];
            body.lh = p.last_h + p.last_off[h];
            body.le = p.last_e + p.last_off[h];
            body.hit_i = INT_MAX;
            body.hit_j = INT_MAX;
            body.cand = INT_MAX;
            body.rr = ResidueRing{ grp.sh->residues[grp.wig], 0, p.db.codes + p.db.offsets[hit.id], (int32_t) body.B,
                                   rg.b_end };
            run_stripes<W>( body, *grp.sh, grp.gb, grp.wig, grp.lane, (body.A + TB_ROWS - 1) / TB_ROWS, body.B,
                    p.error_flags );
            int32_t bi = body.hit_i, bj = body.hit_j;
            for( int o = 16; o > 0; o >>= 1 ) {
                const int32_t i = __shfl_xor_sync( 0xffffffffu, bi, o );
                const int32_t j = __shfl_xor_sync( 0xffffffffu, bj, o );
                if( i < bi || (i == bi && j < bj) ) {
                    bi = i;
                    bj = j;
                }
            }
            if( grp.lane == 0 ) {
                grp.sh->red[grp.wig][0] = bi;
                grp.sh->red[grp.wig][1] = bj;
            }
            grp.gb.sync();
            if( grp.wig == 0 && grp.lane == 0 ) {
                for( int k = 1; k < W; k++ ) {
                    const int32_t i = grp.sh->red[k][0], j = grp.sh->red[k][1];
                    if( i < bi || (i == bi && j < bj) ) {
                        bi = i;
                        bj = j;
                    }
                }
                if( bi == INT_MAX ) {
                    rg.status = 2;
                }
                else {
                    rg.b_begin = rg.b_end - bi;
                    rg.a_begin = rg.a_end - bj;
                }
                p.regions[h] = rg;
            }
        }
        grp.gb.sync();
    }
}

// ---------------------------------------------------------------------------
// 3. Direction pass (reference: src/algo/cigar.c:48-198).  Query rows on
//    lanes, database columns streamed, exactly the reference orientation.
//    Codes: 0 = M, 1 = D (UP|EXT_UP), 2 = I (LEFT|EXT_LEFT, takes priority).
//    Stored for columns [b_begin, b_end] and all query rows of the lane, one
//    16-bit word (8 rows x 2 bits) per lane and column.
// ---------------------------------------------------------------------------
template <int W>
struct DirectionStripe : TbStripeBase<W> {
    static constexpr int32_t cand = INT32_MAX;
    const uint8_t * a;
    uint32_t A, B, words;
    bool nw;
    int32_t b_begin;
    uint16_t * dir;
    int32_t * corner;              // Needleman-Wunsch: receives H(A - 1, B - 1)

    __device__ void begin( uint32_t stripe ) {
        const int32_t gO = this->gO, gE = this->gE;
        this->link.stripe = stripe;
        this->link.last = (stripe + 1) * TB_ROWS >= A;
        this->row0 = (int32_t) (stripe * TB_ROWS) + this->lane * TB_R;
        const int32_t row0 = this->row0;
        this->nvalid = max( 0, min( TB_R, (int) A - row0 ) );
        load_rows( a, row0, 1, this->nvalid, this->qa );
#pragma unroll
        for( int r = 0; r < TB_R; r++ ) {
            const int32_t i = row0 + r;
            this->H[r] = nw ? gO + (i + 1) * gE : 0;
            this->E[r] = nw ? 2 * gO + (i + 2) * gE : 0;
        }
        this->diag = nw ? ((row0 == 0) ? 0 : gO + row0 * gE) : 0;
        this->out_h = 0;
        this->out_f = 0;
        this->link.start( B, this->lane );
        this->rr.start( this->lane );
    }

    __device__ bool chunk( uint32_t ck, int32_t ) {
        const uint32_t steps = B + 31, s0 = ck * 32;
        const int lane = this->lane;
        const int32_t gO = this->gO, gE = this->gE, gOE = this->gOE;
        const int32_t row0 = this->row0;
        // one wavefront step; edge: some lane may be on a column outside 0..B-1
        auto column = [&]( const uint32_t s, const bool edge ) {
            int32_t up_h = __shfl_up_sync( 0xffffffffu, this->out_h, 1 );
            int32_t up_f = __shfl_up_sync( 0xffffffffu, this->out_f, 1 );
            const int32_t j = (int32_t) s - lane;     // database index
            if( edge && (j < 0 || j >= (int32_t) B) )
                return;
            // H(-1, j) is the next column's row-0 diagonal
            this->above( s, j, nw ? gO + (j + 1) * gE : 0, nw ? 2 * gO + (j + 2) * gE : 0, up_h, up_f );
            const int d = this->rr.get( s, lane );
            int32_t f = up_f, hd = this->diag;
            uint32_t code = 0;
            // flags as in the reference (strict compares in its order),
            // computed beside a branch-free row-to-row chain
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t e = this->E[r];
                const int32_t x0 = hd + mget( this->smat, d, this->qa[r] );
                // each max also yields the negation of one strict flag
                bool no_up, no_left, no_ext_up, no_ext_left;
                const int32_t m1 = __vibmax_s32( x0, f, &no_up );       // UP: f > x0
                const int32_t xr = __vibmax_s32( m1, e, &no_left );     // LEFT: e > max(x0, f)
                const int32_t x = nw ? xr : max( xr, 0 );
                hd = this->H[r];
                this->H[r] = x;
                const int32_t y = x + gOE;
                f = __vibmax_s32( y, f + gE, &no_ext_up );               // EXT_UP: f + gapE > y
                this->E[r] = __vibmax_s32( y, e + gE, &no_ext_left );    // EXT_LEFT: e + gapE > y
                // rows past the query's end get codes too; the walk never reads them
                const bool ins = !(no_left && no_ext_left);
                const bool del = !(no_up && no_ext_up);
                code |= (ins ? 2u : (del ? 1u : 0u)) << (2 * r);
            }
            this->diag = up_h;
            this->out_h = this->H[TB_R - 1];
            this->out_f = f;
            if( j >= b_begin && (uint32_t) (row0 / TB_R) < words )
                dir[(uint64_t) (j - b_begin) * words + row0 / TB_R] = (uint16_t) code;
            if( nw && j == (int32_t) B - 1 ) {
                // the global score: the last cell of the full matrix
                const int32_t rl = (int32_t) A - 1 - row0;
#pragma unroll
                for( int r = 0; r < TB_R; r++ )
                    if( r == rl )
                        *corner = this->H[r];
            }
            this->put_bottom( j );
        };
        // the residue ring and the boundary prefetch refill at the first step of a chunk
        this->link.step( B, s0, lane );
        this->rr.step( s0, lane );
        const uint32_t s1 = min( s0 + 32, steps );
        if( s0 >= 31 && s1 <= B ) {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, false );
        }
        else {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, true );
        }
        return s0 + 32 < steps;
    }

    __device__ void end() {}
};

template <int W>
__global__ void __launch_bounds__( 256 ) tb_directions_kernel( TbParams p ) {
    __shared__ PipeShared<W> shs[TbGroup<W>::GROUPS];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, false );
    TbGroup<W> grp( shs, p );
    for( ;; ) {
        const uint32_t h = grp.take( p.hit_counters + 2 );
        if( h >= p.n_hits )
            break;
        const TbHit hit = p.hits[h];
        const TbRegion rg = p.regions[h];
        if( rg.status == 0 ) {
            DirectionStripe<W> body;
            grp.link( body, smat, p );
            body.nw = hit.algo == 1;
            body.A = (uint32_t) rg.a_end + 1;   // rows 0..a_end suffice
            body.B = (uint32_t) rg.b_end + 1;   // columns 0..b_end
            body.words = (body.A + TB_R - 1) / TB_R;
            body.b_begin = rg.b_begin;
            body.a = p.qcodes + p.qoff[hit.qslot];
            body.dir = p.dirs + p.dir_off[h];
            body.corner = &p.regions[h].fwd_score;
            body.rr = ResidueRing{ grp.sh->residues[grp.wig], 0, p.db.codes + p.db.offsets[hit.id], (int32_t) body.B,
                                   -1 };
            run_stripes<W>( body, *grp.sh, grp.gb, grp.wig, grp.lane, (body.A + TB_ROWS - 1) / TB_ROWS, body.B,
                    p.error_flags );
        }
        grp.gb.sync();
    }
}

// ---------------------------------------------------------------------------
// 1 + 3 fused (Smith-Waterman, symmetric score table): the forward region pass
//    and the direction pass in one sweep of the whole matrix.  The direction
//    pass's recurrence (reference: src/algo/cigar.c:125-200) and the forward
//    pass's (src/algo/align.c:39-82) give every cell the same H: they differ
//    only in the E and F values that enter the first column and row, which are
//    never above zero and so never reach a Smith-Waterman cell.  With a
//    symmetric table the two orientations score alike.  So this pass computes
//    the direction words with the direction pass's values, the end cell (first
//    maximum, database index then query index) from H, and the last column's H
//    and E for the reverse pass.  That E is the forward pass's: at the last
//    column the E chain from earlier cells is at least gapO + gapE (H >= 0),
//    and the host runs this pass only where (B - 1) x gapE < gapO + gapE, so
//    neither pass's initial term can be the maximum there.  Directions are
//    stored for every column and every query row.
// ---------------------------------------------------------------------------
template <int W>
struct FwdDirStripe : TbStripeBase<W> {
    static constexpr int32_t cand = INT32_MAX;
    const uint8_t * a;
    uint32_t A, B, words;
    uint16_t * dir;
    int32_t * lh;
    int32_t * le;
    int32_t pv, pi, pj;                       // this stripe's first maximum
    int32_t best_v, best_i, best_j;           // over the warp's stripes

    __device__ void begin( uint32_t stripe ) {
        this->link.stripe = stripe;
        this->link.last = (stripe + 1) * TB_ROWS >= A;
        this->row0 = (int32_t) (stripe * TB_ROWS) + this->lane * TB_R;
        this->nvalid = max( 0, min( TB_R, (int) A - this->row0 ) );
        load_rows( a, this->row0, 1, this->nvalid, this->qa );
#pragma unroll
        for( int r = 0; r < TB_R; r++ ) {
            this->H[r] = 0;
            this->E[r] = 0;
        }
        this->diag = 0;
        this->out_h = 0;
        this->out_f = 0;
        pv = 0;
        pi = INT_MAX;
        pj = INT_MAX;
        this->link.start( B, this->lane );
        this->rr.start( this->lane );
    }

    __device__ bool chunk( uint32_t ck, int32_t ) {
        const uint32_t steps = B + 31, s0 = ck * 32;
        const int lane = this->lane;
        const int32_t gE = this->gE, gOE = this->gOE;
        const int32_t row0 = this->row0;
        // one wavefront step; edge: some lane may be on a column outside 0..B-1
        auto column = [&]( const uint32_t s, const bool edge ) {
            int32_t up_h = __shfl_up_sync( 0xffffffffu, this->out_h, 1 );
            int32_t up_f = __shfl_up_sync( 0xffffffffu, this->out_f, 1 );
            const int32_t j = (int32_t) s - lane;     // database index
            if( edge && (j < 0 || j >= (int32_t) B) )
                return;
            this->above( s, j, 0, 0, up_h, up_f );
            const int d = this->rr.get( s, lane );
            int32_t f = up_f, hd = this->diag;
            uint32_t code = 0;
            int32_t e_last[TB_R];
#pragma unroll
            for( int r = 0; r < TB_R; r++ ) {
                const int32_t e = this->E[r];
                const int32_t x0 = hd + mget( this->smat, d, this->qa[r] );
                bool no_up, no_left, no_ext_up, no_ext_left;
                const int32_t m1 = __vibmax_s32( x0, f, &no_up );       // UP: f > x0
                const int32_t xr = __vibmax_s32( m1, e, &no_left );     // LEFT: e > max(x0, f)
                const int32_t x = max( xr, 0 );
                // the lane visits its cells in (column, row) order: within a
                // stripe the first maximum wins with a strict compare
                const bool take = (r < this->nvalid) && x > pv;
                pv = take ? x : pv;
                pi = take ? j : pi;
                pj = take ? row0 + r : pj;
                e_last[r] = e;
                hd = this->H[r];
                this->H[r] = x;
                const int32_t y = x + gOE;
                f = __vibmax_s32( y, f + gE, &no_ext_up );               // EXT_UP: f + gapE > y
                this->E[r] = __vibmax_s32( y, e + gE, &no_ext_left );    // EXT_LEFT: e + gapE > y
                // rows past the query's end get codes too; the walk never reads them
                const bool ins = !(no_left && no_ext_left);
                const bool del = !(no_up && no_ext_up);
                code |= (ins ? 2u : (del ? 1u : 0u)) << (2 * r);
            }
            if( (uint32_t) (row0 / TB_R) < words )
                dir[(uint64_t) j * words + row0 / TB_R] = (uint16_t) code;
            if( j == (int32_t) B - 1 ) {
#pragma unroll
                for( int r = 0; r < TB_R; r++ )
                    if( r < this->nvalid ) {
                        lh[row0 + r] = this->H[r];
                        le[row0 + r] = e_last[r];
                    }
            }
            this->diag = up_h;
            this->out_h = this->H[TB_R - 1];
            this->out_f = f;
            this->put_bottom( j );
        };
        // the residue ring and the boundary prefetch refill at the first step of a chunk
        this->link.step( B, s0, lane );
        this->rr.step( s0, lane );
        const uint32_t s1 = min( s0 + 32, steps );
        if( s0 >= 31 && s1 <= B ) {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, false );
        }
        else {
            for( uint32_t s = s0; s < s1; s++ )
                column( s, true );
        }
        return s0 + 32 < steps;
    }

    // this stripe's first maximum against the earlier stripes' (value desc,
    // database index asc, query index asc)
    __device__ void end() {
        if( pv > best_v || (pv == best_v && pv > 0 && (pi < best_i || (pi == best_i && pj < best_j))) ) {
            best_v = pv;
            best_i = pi;
            best_j = pj;
        }
    }
};

template <int W>
__global__ void __launch_bounds__( 256 ) tb_fwddir_kernel( TbParams p ) {
    __shared__ PipeShared<W> shs[TbGroup<W>::GROUPS];
    __shared__ int32_t smat[1024];
    stage_matrix( p.matrix, smat, false );
    TbGroup<W> grp( shs, p );
    for( ;; ) {
        const uint32_t h = grp.take( p.hit_counters + 0 );
        if( h >= p.n_hits )
            break;
        const TbHit hit = p.hits[h];
        FwdDirStripe<W> body;
        grp.link( body, smat, p );
        body.A = p.qlen[hit.qslot];
        body.B = p.db.lens[hit.id];
        body.words = (body.A + TB_R - 1) / TB_R;
        body.a = p.qcodes + p.qoff[hit.qslot];
        body.dir = p.dirs + p.dir_off[h];
        body.lh = p.last_h + p.last_off[h];
        body.le = p.last_e + p.last_off[h];
        body.best_v = 0;
        body.best_i = INT_MAX;
        body.best_j = INT_MAX;
        body.rr = ResidueRing{ grp.sh->residues[grp.wig], 0, p.db.codes + p.db.offsets[hit.id], (int32_t) body.B, -1 };
        run_stripes<W>( body, *grp.sh, grp.gb, grp.wig, grp.lane, (body.A + TB_ROWS - 1) / TB_ROWS, body.B,
                p.error_flags );
        // the best key over the warp, then over the group
        int32_t bv = body.best_v, bi = body.best_i, bj = body.best_j;
        for( int o = 16; o > 0; o >>= 1 ) {
            const int32_t v = __shfl_xor_sync( 0xffffffffu, bv, o );
            const int32_t i = __shfl_xor_sync( 0xffffffffu, bi, o );
            const int32_t j = __shfl_xor_sync( 0xffffffffu, bj, o );
            if( v > bv || (v == bv && (i < bi || (i == bi && j < bj))) ) {
                bv = v;
                bi = i;
                bj = j;
            }
        }
        if( grp.lane == 0 ) {
            grp.sh->red[grp.wig][0] = bv;
            grp.sh->red[grp.wig][1] = bi;
            grp.sh->red[grp.wig][2] = bj;
        }
        grp.gb.sync();
        if( grp.wig == 0 && grp.lane == 0 ) {
            for( int k = 1; k < W; k++ ) {
                const int32_t v = grp.sh->red[k][0], i = grp.sh->red[k][1], j = grp.sh->red[k][2];
                if( v > bv || (v == bv && (i < bi || (i == bi && j < bj))) ) {
                    bv = v;
                    bi = i;
                    bj = j;
                }
            }
            // the host set the direction layout of the region; keep it
            TbRegion rg = p.regions[h];
            rg.fwd_score = bv;
            rg.a_end = bj;
            rg.b_end = bi;
            rg.a_begin = 0;
            rg.b_begin = 0;
            rg.status = (bv > 0) ? 0 : 1;
            p.regions[h] = rg;
        }
        // every warp is past this hit's shared state before the next hit
        grp.gb.sync();
    }
}

// ---------------------------------------------------------------------------
// 4. Walk (reference: src/algo/cigar.c:300-334): one warp per hit writes the
//    moves in traceback order (end to begin); the host run-length encodes.
//    Each step reads the direction word of the current cell, which the
//    previous step chose, so a walk that reads HBM or L2 word by word waits a
//    memory round trip per move.  In 32 moves the path stays within 32 rows
//    and 32 columns of its current cell (every move leaves the row or the
//    column or both by one), so the warp loads that window (32 columns, at
//    most 5 words of 8 rows each) into shared memory with one load round,
//    lane 0 walks up to 32 moves from it, and the warp loads the next window.
// ---------------------------------------------------------------------------
constexpr int TB_WALK_WARPS = 4;                 // hits per CTA
constexpr int TB_WALK_WORDS = 32 / TB_R + 1;     // direction words a 32-row window spans

__global__ void __launch_bounds__( 32 * TB_WALK_WARPS ) tb_walk_kernel( TbParams p ) {
    __shared__ uint16_t win[TB_WALK_WARPS][32][TB_WALK_WORDS];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t h = blockIdx.x * TB_WALK_WARPS + (uint32_t) wib;
    if( h >= p.n_hits )
        return;                                  // the whole warp
    const TbRegion rg = p.regions[h];
    if( rg.status != 0 ) {
        if( lane == 0 )
            p.ops_len[h] = 0;
        return;
    }
    const uint32_t words = (uint32_t) rg.dir_words;
    const uint16_t * dir = p.dirs + p.dir_off[h];
    char * out = p.ops + p.ops_off[h];
    const uint64_t cap = p.ops_off[h + 1] - p.ops_off[h];
    const int64_t a_begin = rg.a_begin, b_begin = rg.b_begin;
    const int64_t j_lo = max( b_begin, (int64_t) rg.dir_col0 );   // columns held in the layout
    int64_t i = rg.a_end, j = rg.b_end;
    uint64_t n = 0;
    while( i >= a_begin && j >= b_begin && i >= 0 && j >= 0 ) {
        // the window: columns j - 31 .. j, words of rows max(i - 31, 0) .. i
        const int64_t w0 = max( i - 31, (int64_t) 0 ) / TB_R;
        const int64_t jc = j - lane;
#pragma unroll
        for( int k = 0; k < TB_WALK_WORDS; k++ ) {
            const int64_t w = w0 + k;
            uint16_t v = 0;
            if( jc >= j_lo && w <= i / TB_R && w < (int64_t) words )
                v = dir[(uint64_t) (jc - rg.dir_col0) * words + (uint64_t) w];
            win[wib][lane][k] = v;
        }
        __syncwarp();
        if( lane == 0 ) {
            const int64_t j0 = j;
            for( int m = 0; m < 32 && i >= a_begin && j >= b_begin && i >= 0 && j >= 0; m++ ) {
                const uint32_t word = win[wib][j0 - j][i / TB_R - w0];
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
        }
        i = __shfl_sync( 0xffffffffu, i, 0 );
        j = __shfl_sync( 0xffffffffu, j, 0 );
        n = __shfl_sync( 0xffffffffu, n, 0 );
        __syncwarp();
    }
    if( lane == 0 )
        p.ops_len[h] = (uint32_t) n;
}

static void launch_walk( const TbParams & p, cudaStream_t st ) {
    tb_walk_kernel<<<(p.n_hits + TB_WALK_WARPS - 1) / TB_WALK_WARPS, 32 * TB_WALK_WARPS, 0, st>>>( p );
}

// Region phase (Smith-Waterman hits only): forward and reverse passes.  They
// need no direction memory, so all hits of a search run in one launch each.
// group: warps per hit (1, 2 or 4).  ev (optional): 3 events recorded around
// the two kernels.
cudaError_t launch_tb_regions( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev ) {
    if( ev )
        cudaEventRecord( ev[0], st );
    if( p.n_hits ) {
        if( group == 4 )
            tb_forward_kernel<4><<<grid, 256, 0, st>>>( p );
        else if( group == 2 )
            tb_forward_kernel<2><<<grid, 256, 0, st>>>( p );
        else
            tb_forward_kernel<1><<<grid, 256, 0, st>>>( p );
        if( ev )
            cudaEventRecord( ev[1], st );
        if( group == 4 )
            tb_reverse_kernel<4><<<grid, 256, 0, st>>>( p );
        else if( group == 2 )
            tb_reverse_kernel<2><<<grid, 256, 0, st>>>( p );
        else
            tb_reverse_kernel<1><<<grid, 256, 0, st>>>( p );
    }
    else if( ev ) {
        cudaEventRecord( ev[1], st );
    }
    if( ev )
        cudaEventRecord( ev[2], st );
    return cudaGetLastError();
}

// Fused Smith-Waterman traceback of the hits of one wave: the forward region
// pass with the direction words (symmetric score table), the reverse pass and
// the walk.  ev (optional): 3 events, before and after the fused pass and after
// the walk.
cudaError_t launch_tb_fused( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev ) {
    if( ev )
        cudaEventRecord( ev[0], st );
    if( p.n_hits ) {
        if( group == 4 ) {
            tb_fwddir_kernel<4><<<grid, 256, 0, st>>>( p );
            if( ev )
                cudaEventRecord( ev[1], st );
            tb_reverse_kernel<4><<<grid, 256, 0, st>>>( p );
        }
        else if( group == 2 ) {
            tb_fwddir_kernel<2><<<grid, 256, 0, st>>>( p );
            if( ev )
                cudaEventRecord( ev[1], st );
            tb_reverse_kernel<2><<<grid, 256, 0, st>>>( p );
        }
        else {
            tb_fwddir_kernel<1><<<grid, 256, 0, st>>>( p );
            if( ev )
                cudaEventRecord( ev[1], st );
            tb_reverse_kernel<1><<<grid, 256, 0, st>>>( p );
        }
        launch_walk( p, st );
    }
    else if( ev ) {
        cudaEventRecord( ev[1], st );
    }
    if( ev )
        cudaEventRecord( ev[2], st );
    return cudaGetLastError();
}

// Path phase: direction pass and walk of the hits of one wave (the hits whose
// direction words fit the memory the host set aside).  ev (optional): 3 events
// recorded around the two kernels.
cudaError_t launch_tb_paths( const TbParams & p, int group, int grid, cudaStream_t st, cudaEvent_t * ev ) {
    if( ev )
        cudaEventRecord( ev[0], st );
    if( p.n_hits ) {
        if( group == 4 )
            tb_directions_kernel<4><<<grid, 256, 0, st>>>( p );
        else if( group == 2 )
            tb_directions_kernel<2><<<grid, 256, 0, st>>>( p );
        else
            tb_directions_kernel<1><<<grid, 256, 0, st>>>( p );
        if( ev )
            cudaEventRecord( ev[1], st );
        launch_walk( p, st );
    }
    else if( ev ) {
        cudaEventRecord( ev[1], st );
    }
    if( ev )
        cudaEventRecord( ev[2], st );
    return cudaGetLastError();
}

}  // namespace ssa
