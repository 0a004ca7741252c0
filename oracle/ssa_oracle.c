/*
 * ssa_oracle.c -- CPU restatement of the libssa database-search path.
 *
 * TEST INFRASTRUCTURE ONLY (see ssa_oracle.h).  This is deliberately a slow,
 * literal emulation: every SIMD lane of the reference's inter-sequence kernels
 * is simulated with scalar saturating arithmetic, block by block, with the
 * reference's channel scheduler deciding which database sequence enters which
 * lane and when its score reaches the heap.  It is the ground truth for the
 * hit order including ties, and is itself checked against the reference
 * binary (oracle/_ref/ref_run) by the tests.
 */
#include "ssa_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define CDEPTH 4

static int64_t max64( int64_t a, int64_t b ) { return a > b ? a : b; }
static int64_t min64( int64_t a, int64_t b ) { return a < b ? a : b; }

/* Saturating clamp to a signed width (8 or 16 bits); 64 means no clamp. */
static int64_t sat( int64_t x, int w ) {
    if( w == 64 )
        return x;
    int64_t lo = -((int64_t) 1 << (w - 1)), hi = ((int64_t) 1 << (w - 1)) - 1;
    return x < lo ? lo : (x > hi ? hi : x);
}

/* Two's-complement truncation, as assigning an int to int8_t/int16_t. */
static int64_t trunc_w( int64_t x, int w ) {
    if( w == 8 )
        return (int8_t) x;
    if( w == 16 )
        return (int16_t) x;
    return x;
}

static int64_t mat( const oracle_config * cfg, int w, int row, int col ) {
    /* reference: src/matrices.c:372-377 -- the 8/16-bit tables are truncating
     * copies of the 64-bit table */
    return trunc_w( cfg->matrix[(row << 5) + col], w );
}

/* ------------------------------------------------------------------------ */
/* Min-heap of the top hits (reference: src/util/minheap.c:50-91).          */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint64_t db_id;
    int64_t score;
} elem;

typedef struct {
    uint64_t alloc, count;
    elem * a;
} heap;

static void heap_add( heap * m, uint64_t id, int64_t score ) {
    elem n = { id, score };
    if( m->alloc == 0 )
        return;
    if( m->count < m->alloc ) {
        /* sift up while strictly smaller than the parent (minheap.c:77-86) */
        uint64_t i = m->count++;
        while( i > 0 && n.score < m->a[(i - 1) / 2].score ) {
            m->a[i] = m->a[(i - 1) / 2];
            i = (i - 1) / 2;
        }
        m->a[i] = n;
    }
    else if( m->a[0].score < n.score ) {
        /* replace the root only when strictly greater (minheap.c:87-90, 50-73) */
        uint64_t p = 0, c = 1;
        while( c < m->count ) {
            if( c + 1 < m->count && m->a[c + 1].score < m->a[c].score )
                c++;
            if( m->a[c].score < n.score )
                m->a[p] = m->a[c];
            else
                break;
            p = c;
            c = 2 * p + 1;
        }
        m->a[p] = n;
    }
}

/* qsort by score, then ID, both descending (minheap.c:93-106, util.h:31). */
static int elem_cmp( const void * x, const void * y ) {
    const elem * a = x, * b = y;
    if( a->score != b->score )
        return a->score > b->score ? -1 : 1;
    if( a->db_id != b->db_id )
        return a->db_id > b->db_id ? -1 : 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exact scalar kernels.                                                    */
/* ------------------------------------------------------------------------ */
int64_t oracle_full_sw( const oracle_config * cfg, const uint8_t * dseq, uint64_t dlen, const uint8_t * q,
        uint64_t qlen ) {
    /* reference: src/algo/64/smith_waterman_63.c:32-98 */
    int64_t gO = cfg->gap_open, gE = cfg->gap_extend;
    int64_t * hh = calloc( qlen ? qlen : 1, sizeof(int64_t) );
    int64_t * ee = calloc( qlen ? qlen : 1, sizeof(int64_t) );
    int64_t s = 0;
    for( uint64_t j = 0; j < dlen; j++ ) {
        int64_t f = 0, h = 0;
        for( uint64_t i = 0; i < qlen; i++ ) {
            int64_t n = hh[i], e = ee[i];
            h += cfg->matrix[(dseq[j] << 5) + q[i]];
            if( e > h ) h = e;
            if( f > h ) h = f;
            if( h < 0 ) h = 0;
            if( h > s ) s = h;
            hh[i] = h;
            e += gE;
            f += gE;
            h += gO + gE;
            if( h > e ) e = h;
            if( h > f ) f = h;
            ee[i] = e;
            h = n;
        }
    }
    free( hh );
    free( ee );
    return s;
}

int64_t oracle_full_nw( const oracle_config * cfg, const uint8_t * dseq, uint64_t dlen, const uint8_t * q,
        uint64_t qlen ) {
    /* reference: src/algo/64/needleman_wunsch_64.c:32-98 */
    int64_t gO = cfg->gap_open, gE = cfg->gap_extend;
    int64_t * hh = malloc( (qlen ? qlen : 1) * sizeof(int64_t) );
    int64_t * ee = malloc( (qlen ? qlen : 1) * sizeof(int64_t) );
    for( uint64_t i = 0; i < qlen; i++ ) {
        hh[i] = gO + (int64_t) (i + 1) * gE;
        ee[i] = 2 * gO + (int64_t) (i + 2) * gE;
    }
    for( uint64_t j = 0; j < dlen; j++ ) {
        int64_t f = 2 * gO + (int64_t) (j + 2) * gE;
        int64_t h = (j == 0) ? 0 : (gO + (int64_t) j * gE);
        for( uint64_t i = 0; i < qlen; i++ ) {
            int64_t n = hh[i], e = ee[i];
            h += cfg->matrix[(dseq[j] << 5) + q[i]];
            if( f > h ) h = f;
            if( e > h ) h = e;
            hh[i] = h;
            e += gE;
            f += gE;
            h += gO + gE;
            if( f < h ) f = h;
            if( e < h ) e = h;
            ee[i] = e;
            h = n;
        }
    }
    int64_t r = qlen ? hh[qlen - 1] : 0;
    free( hh );
    free( ee );
    return r;
}

/* ------------------------------------------------------------------------ */
/* Saturating inter-sequence pass with the channel scheduler.               */
/* reference: src/algo/simd/search_simd_sw.c:172-441 (SW) and               */
/*            src/algo/simd/search_simd_nw.c:180-516 (NW)                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint64_t idx;           /* index into the pass's sequence list, or UINT64_MAX */
    uint64_t pos, len;      /* residues consumed / total */
    int win[CDEPTH];        /* current 4-residue window (0 = pad) */
    int ovf;
    int64_t S;              /* SW running maximum */
    int64_t hmin, hmax;     /* NW block extrema since the last change block */
    int64_t Hb[CDEPTH], Fb[CDEPTH];   /* NW top-boundary carries */
    int64_t Sm[CDEPTH];     /* NW last-row values of the last block */
    int64_t blocks;
    int64_t * H, * E;       /* per-query-row column state */
} lane_t;

typedef struct {
    int algo, w, lanes;
    const oracle_config * cfg;
    const uint8_t * q;
    uint64_t qlen;
    int64_t gOE, gE, thresh, MIN, MAX;
} pass_t;

static void pass_init( pass_t * p, const oracle_config * cfg, int w, int lanes, const uint8_t * q, uint64_t qlen ) {
    p->algo = cfg->algo;
    p->w = w;
    p->lanes = lanes;
    p->cfg = cfg;
    p->q = q;
    p->qlen = qlen;
    p->MIN = -((int64_t) 1 << (w - 1));
    p->MAX = ((int64_t) 1 << (w - 1)) - 1;
    /* set1_epi8/16 of an int expression truncates (search_simd_sw.c:319-320,
     * search_simd_nw.c:360-361, 372) */
    p->gOE = trunc_w( cfg->gap_open + cfg->gap_extend, w );
    p->gE = trunc_w( cfg->gap_extend, w );
    p->thresh = trunc_w( p->MIN - cfg->gap_open - cfg->gap_extend - 1, w );
}

/* Loads the next CDEPTH residues of a lane; returns 1 when the sequence is
 * exhausted after this load (reference: src/algo/8/search_8_util.h:60-74). */
static int move_window( lane_t * l, const uint8_t * seq ) {
    for( int j = 0; j < CDEPTH; j++ )
        l->win[j] = (l->pos < l->len) ? seq[l->pos++] : 0;
    return l->pos == l->len;
}

/* One 4-column block of one lane.  fresh: the lane starts a sequence here
 * (the M mask).  first: the block is a change block. */
static void lane_block( const pass_t * p, lane_t * l, int fresh, int first ) {
    const int w = p->w;
    const int64_t MIN = p->MIN, gOE = p->gOE, gE = p->gE;
    int64_t h[CDEPTH], f[CDEPTH], n[CDEPTH];
    int64_t v[CDEPTH];
    if( p->algo == 0 ) {
        /* aligncolumns_first/rest, search_simd_sw.c:184-277 */
        for( int k = 0; k < CDEPTH; k++ ) {
            h[k] = MIN;
            f[k] = MIN;
        }
        for( uint64_t i = 0; i < p->qlen; i++ ) {
            int64_t h4 = l->H[i], e = l->E[i];
            if( fresh ) {
                h4 = MIN;
                e = MIN;
            }
            for( int k = 0; k < CDEPTH; k++ )
                v[k] = mat( p->cfg, w, l->win[k], p->q[i] );
            for( int k = 0; k < CDEPTH; k++ ) {
                int64_t x = sat( h[k] + v[k], w );
                x = max64( x, f[k] );
                x = max64( x, e );
                l->S = max64( l->S, x );
                n[k] = x;
                x = sat( x + gOE, w );
                f[k] = max64( sat( f[k] + gE, w ), x );
                e = max64( sat( e + gE, w ), x );
            }
            l->H[i] = n[3];
            l->E[i] = e;
            h[0] = h4;
            h[1] = n[0];
            h[2] = n[1];
            h[3] = n[2];
        }
    }
    else {
        /* aligncolumns_first/rest, search_simd_nw.c:193-312 */
        if( first ) {
            l->hmin = 0;
            l->hmax = 0;
        }
        for( int k = 0; k < CDEPTH; k++ ) {
            f[k] = sat( l->Fb[k] + gOE, w );
            h[k] = l->Hb[k];
        }
        int64_t mge = fresh ? gOE : 0;
        const int64_t mgoe = fresh ? gOE : 0, mgext = fresh ? gE : 0;
        for( uint64_t i = 0; i < p->qlen; i++ ) {
            int64_t h4 = l->H[i], e = l->E[i];
            if( first ) {
                if( fresh ) {
                    h4 = 0;
                    e = 0;
                }
                h4 = sat( h4 + mge, w );
                e = sat( e + mge, w );
                e = sat( e + mgoe, w );
                mge = sat( mge + mgext, w );
            }
            for( int k = 0; k < CDEPTH; k++ )
                v[k] = mat( p->cfg, w, l->win[k], p->q[i] );
            for( int k = 0; k < CDEPTH; k++ ) {
                int64_t x = sat( h[k] + v[k], w );
                x = max64( x, f[k] );
                x = max64( x, e );
                l->hmin = min64( l->hmin, x );
                l->hmax = max64( l->hmax, x );
                n[k] = x;
                x = sat( x + gOE, w );
                f[k] = max64( sat( f[k] + gE, w ), x );
                e = max64( sat( e + gE, w ), x );
            }
            l->H[i] = n[3];
            l->E[i] = e;
            h[0] = h4;
            h[1] = n[0];
            h[2] = n[1];
            h[3] = n[2];
            if( i + 1 == p->qlen )
                for( int k = 0; k < CDEPTH; k++ )
                    l->Sm[k] = n[k];
        }
    }
    l->blocks++;
}

static int lane_overflowed( const pass_t * p, const lane_t * l ) {
    if( p->algo == 0 )
        return l->S == p->MAX; /* search_simd_sw.c:422-423 */
    return (l->hmin < p->thresh) || (l->hmax == p->MAX); /* search_simd_nw.c:483-485 */
}

static void lane_nw_carry( const pass_t * p, lane_t * l ) {
    /* search_simd_nw.c:494-502 */
    l->Fb[0] = sat( l->Fb[3] + p->gE, p->w );
    l->Fb[1] = sat( l->Fb[0] + p->gE, p->w );
    l->Fb[2] = sat( l->Fb[1] + p->gE, p->w );
    l->Fb[3] = sat( l->Fb[2] + p->gE, p->w );
    l->Hb[0] = sat( l->Hb[3] + p->gE, p->w );
    l->Hb[1] = sat( l->Hb[0] + p->gE, p->w );
    l->Hb[2] = sat( l->Hb[1] + p->gE, p->w );
    l->Hb[3] = sat( l->Hb[2] + p->gE, p->w );
}

static void lane_start_nw( const pass_t * p, lane_t * l ) {
    /* search_simd_nw.c:445-453: integer expressions truncated to the width */
    int64_t gO = p->cfg->gap_open, gE = p->cfg->gap_extend;
    l->Hb[0] = 0;
    l->Hb[1] = trunc_w( gO + 1 * gE, p->w );
    l->Hb[2] = trunc_w( gO + 2 * gE, p->w );
    l->Hb[3] = trunc_w( gO + 3 * gE, p->w );
    l->Fb[0] = trunc_w( gO + 1 * gE, p->w );
    l->Fb[1] = trunc_w( gO + 2 * gE, p->w );
    l->Fb[2] = trunc_w( gO + 3 * gE, p->w );
    l->Fb[3] = trunc_w( gO + 4 * gE, p->w );
}

typedef struct {
    uint64_t n;
    uint64_t * ids;         /* database IDs */
    const uint8_t ** seqs;
    uint64_t * lens;
} seqlist;

/* Callback sinks of a pass: reported scores go to the heap, overflowed
 * sequences to the next pass's list, both in report order. */
typedef struct {
    heap * hp;
    seqlist * ovf;
} sink_t;

/* reference: search_YY_XXX_sw (search_simd_sw.c:279-441) and
 * search_YY_XXX_nw (search_simd_nw.c:314-516): the block loop and channel
 * scheduler, restated for C lanes of scalar state. */
static void run_pass( const pass_t * p, const seqlist * in, sink_t * sink, uint64_t * rep_blocks ) {
    const int C = p->lanes;
    lane_t * L = calloc( C, sizeof(lane_t) );
    int64_t * hbuf = calloc( 2 * (size_t) C * (p->qlen ? p->qlen : 1), sizeof(int64_t) );
    for( int c = 0; c < C; c++ ) {
        L[c].idx = UINT64_MAX;
        L[c].H = hbuf + 2 * (size_t) c * p->qlen;
        L[c].E = L[c].H + p->qlen;
        L[c].S = p->MIN;
    }
    int * fresh = calloc( C, sizeof(int) );
    uint64_t next_id = 0, done = 0;
    int change = 1;
    for( ;; ) {
        int first = change;
        if( !change ) {
            for( int c = 0; c < C; c++ )
                if( L[c].idx != UINT64_MAX )
                    change |= move_window( &L[c], in->seqs[L[c].idx] );
            for( int c = 0; c < C; c++ )
                fresh[c] = 0;
        }
        else {
            change = 0;
            for( int c = 0; c < C; c++ ) {
                fresh[c] = 0;
                if( !L[c].ovf && L[c].idx != UINT64_MAX && L[c].pos < L[c].len ) {
                    change |= move_window( &L[c], in->seqs[L[c].idx] );
                    continue;
                }
                fresh[c] = 1;
                if( L[c].idx != UINT64_MAX ) {
                    uint64_t k = L[c].idx;
                    int64_t score;
                    int ok;
                    if( p->algo == 0 ) {
                        score = L[c].S - p->MIN;
                        ok = !L[c].ovf && score < ((int64_t) 1 << p->w) - 1;
                    }
                    else {
                        score = L[c].Sm[(L[c].len + 3) % 4];
                        ok = !L[c].ovf && score > p->MIN && score < p->MAX;
                    }
                    if( rep_blocks )
                        rep_blocks[k] = (uint64_t) L[c].blocks;
                    if( ok ) {
                        heap_add( sink->hp, in->ids[k], score );
                    }
                    else {
                        seqlist * o = sink->ovf;
                        o->ids[o->n] = in->ids[k];
                        o->seqs[o->n] = in->seqs[k];
                        o->lens[o->n] = in->lens[k];
                        o->n++;
                    }
                    done++;
                }
                if( p->algo == 0 )
                    L[c].S = p->MIN;
                if( next_id < in->n ) {
                    L[c].idx = next_id++;
                    L[c].pos = 0;
                    L[c].len = in->lens[L[c].idx];
                    L[c].blocks = 0;
                    if( p->algo == 1 )
                        lane_start_nw( p, &L[c] );
                    change |= move_window( &L[c], in->seqs[L[c].idx] );
                }
                else {
                    L[c].idx = UINT64_MAX;
                    L[c].pos = L[c].len = 0;
                    for( int j = 0; j < CDEPTH; j++ )
                        L[c].win[j] = 0;
                }
            }
            if( done == in->n )
                break;
        }
        for( int c = 0; c < C; c++ )
            lane_block( p, &L[c], fresh[c], first );
        for( int c = 0; c < C; c++ ) {
            L[c].ovf = lane_overflowed( p, &L[c] );
            change |= L[c].ovf;
            if( p->algo == 1 )
                lane_nw_carry( p, &L[c] );
        }
    }
    free( fresh );
    free( hbuf );
    free( L );
}

oracle_lane oracle_lane_result( const oracle_config * cfg, int width, const uint8_t * query, uint64_t qlen,
        const uint8_t * dseq, uint64_t dlen ) {
    oracle_lane r = { 0, 0, 0 };
    if( width == 64 ) {
        r.score = cfg->algo == 0 ? oracle_full_sw( cfg, dseq, dlen, query, qlen )
                                 : oracle_full_nw( cfg, dseq, dlen, query, qlen );
        return r;
    }
    pass_t p;
    pass_init( &p, cfg, width, 1, query, qlen );
    elem e[1];
    heap hp = { 1, 0, e };
    uint64_t oid[1];
    const uint8_t * os[1];
    uint64_t ol[1];
    seqlist ovf = { 0, oid, os, ol };
    uint64_t id0 = 0;
    const uint8_t * s0 = dseq;
    uint64_t l0 = dlen;
    seqlist in = { 1, &id0, &s0, &l0 };
    sink_t sink = { &hp, &ovf };
    uint64_t blocks = 0;
    run_pass( &p, &in, &sink, &blocks );
    r.overflow = ovf.n > 0;
    r.score = hp.count ? hp.a[0].score : 0;
    r.blocks = (int64_t) blocks;
    return r;
}

/* ------------------------------------------------------------------------ */
/* Traceback (reference: src/algo/align.c:39-182, src/algo/cigar.c:48-346)  */
/* ------------------------------------------------------------------------ */
#define MASK_GAP_UP 1
#define MASK_GAP_LEFT 2
#define MASK_GAP_EXT_UP 4
#define MASK_GAP_EXT_LEFT 8

typedef struct {
    uint64_t a_begin, a_end, b_begin, b_end;
    int ok;
} region_t;

static region_t region_local( const oracle_config * cfg, const uint8_t * a, uint64_t alen, const uint8_t * b,
        uint64_t blen ) {
    /* reference: src/algo/align.c:39-139.  a = query, b = database; the score
     * table is read as [query][db] here (align.c:64,106). */
    region_t r = { 0, 0, 0, 0, 0 };
    int64_t gO = cfg->gap_open, gE = cfg->gap_extend;
    uint64_t size = alen > blen ? alen : blen;
    int64_t * HH = malloc( (size ? size : 1) * sizeof(int64_t) );
    int64_t * EE = malloc( (size ? size : 1) * sizeof(int64_t) );
    int64_t score = 0;
    int found_end = 0;
    for( uint64_t j = 0; j < alen; j++ ) {
        HH[j] = 0;
        EE[j] = gO;
    }
    for( uint64_t i = 0; i < blen; i++ ) {
        int64_t h = 0, p = 0, f = gO;
        for( uint64_t j = 0; j < alen; j++ ) {
            f = max64( f, h + gO ) + gE;
            EE[j] = max64( EE[j], HH[j] + gO ) + gE;
            h = p + cfg->matrix[(a[j] << 5) + b[i]];
            if( h < 0 ) h = 0;
            if( f > h ) h = f;
            if( EE[j] > h ) h = EE[j];
            p = HH[j];
            HH[j] = h;
            if( h > score ) {
                score = h;
                r.a_end = j;
                r.b_end = i;
                found_end = 1;
            }
        }
    }
    if( !found_end ) {
        /* the reference leaves the region uninitialised here (undefined) */
        free( HH );
        free( EE );
        return r;
    }
    /* reverse pass; HH/EE are reset only for indices 0..b_end (align.c:86-89) */
    for( int64_t j = (int64_t) r.b_end; j >= 0; j-- ) {
        HH[j] = -1;
        EE[j] = -1;
    }
    int64_t cost = 0;
    for( int64_t i = (int64_t) r.b_end; i >= 0; i-- ) {
        int64_t h = -1, f = -1;
        int64_t p = (i == (int64_t) r.b_end) ? 0 : -1;
        for( int64_t j = (int64_t) r.a_end; j >= 0; j-- ) {
            f = max64( f, h + gO ) + gE;
            EE[j] = max64( EE[j], HH[j] + gO ) + gE;
            h = p + cfg->matrix[(a[j] << 5) + b[i]];
            if( f > h ) h = f;
            if( EE[j] > h ) h = EE[j];
            p = HH[j];
            HH[j] = h;
            if( h > cost ) {
                cost = h;
                r.a_begin = (uint64_t) j;
                r.b_begin = (uint64_t) i;
                if( cost >= score ) {
                    r.ok = 1;
                    free( HH );
                    free( EE );
                    return r;
                }
            }
        }
    }
    free( HH );
    free( EE );
    return r;
}

static uint8_t * directions( const oracle_config * cfg, const uint8_t * a, uint64_t alen, const uint8_t * b,
        uint64_t blen ) {
    /* reference: src/algo/cigar.c:48-198 */
    int64_t gO = cfg->gap_open, gE = cfg->gap_extend;
    uint8_t * d = calloc( (alen * blen) > 0 ? alen * blen : 1, 1 );
    int64_t * hh = malloc( (alen ? alen : 1) * sizeof(int64_t) );
    int64_t * ee = malloc( (alen ? alen : 1) * sizeof(int64_t) );
    int nw = cfg->algo == 1;
    for( uint64_t i = 0; i < alen; i++ ) {
        hh[i] = nw ? gO + (int64_t) (i + 1) * gE : 0;
        ee[i] = nw ? 2 * gO + (int64_t) (i + 2) * gE : 0;
    }
    for( uint64_t j = 0; j < blen; j++ ) {
        int64_t f = nw ? 2 * gO + (int64_t) (j + 2) * gE : 0;
        int64_t h = nw ? ((j == 0) ? 0 : gO + (int64_t) j * gE) : 0;
        for( uint64_t i = 0; i < alen; i++ ) {
            uint64_t idx = alen * j + i;
            int64_t n = hh[i], e = ee[i];
            h += cfg->matrix[(b[j] << 5) + a[i]];
            if( f > h ) {
                d[idx] |= MASK_GAP_UP;
                h = f;
            }
            if( e > h ) {
                h = e;
                d[idx] |= MASK_GAP_LEFT;
            }
            if( !nw && h < 0 )
                h = 0;
            hh[i] = h;
            h += gO + gE;
            e += gE;
            f += gE;
            if( f > h )
                d[idx] |= MASK_GAP_EXT_UP;
            else
                f = h;
            if( e > h )
                d[idx] |= MASK_GAP_EXT_LEFT;
            else
                e = h;
            ee[i] = e;
            h = n;
        }
    }
    free( hh );
    free( ee );
    return d;
}

int oracle_align_pair( const oracle_config * cfg, const uint8_t * q, uint64_t qlen, const uint8_t * d, uint64_t dlen,
        uint64_t * q_start, uint64_t * q_end, uint64_t * d_start, uint64_t * d_end, char ** cigar ) {
    region_t r;
    if( cfg->algo == 0 ) {
        r = region_local( cfg, q, qlen, d, dlen );
    }
    else {
        r.a_begin = 0;
        r.a_end = qlen - 1;
        r.b_begin = 0;
        r.b_end = dlen - 1;
        r.ok = 1;
    }
    *q_start = r.a_begin;
    *q_end = r.a_end;
    *d_start = r.b_begin;
    *d_end = r.b_end;
    if( !r.ok ) {
        *cigar = calloc( 1, 1 );
        return -1;
    }
    uint8_t * dir = directions( cfg, q, qlen, d, dlen );
    /* traceback with I > D > M priority (cigar.c:300-334) */
    size_t cap = 64, len = 0;
    char * ops = malloc( cap );
    uint64_t i = r.a_end, j = r.b_end;
    while( (i + 1 > 0) && (j + 1 > 0) && (i >= r.a_begin) && (j >= r.b_begin) ) {
        uint8_t x = dir[qlen * j + i];
        char op;
        if( (x & MASK_GAP_LEFT) || (x & MASK_GAP_EXT_LEFT) ) {
            j--;
            op = 'I';
        }
        else if( (x & MASK_GAP_UP) || (x & MASK_GAP_EXT_UP) ) {
            i--;
            op = 'D';
        }
        else {
            i--;
            j--;
            op = 'M';
        }
        if( len + 1 >= cap ) {
            cap *= 2;
            ops = realloc( ops, cap );
        }
        ops[len++] = op;
    }
    free( dir );
    /* run-length encode in alignment order; counts of 1 are not written
     * (cigar.c:221-263) */
    char * out = malloc( len * 21 + 1 );
    size_t o = 0;
    size_t k = len;
    while( k > 0 ) {
        char op = ops[k - 1];
        size_t run = 0;
        while( k > 0 && ops[k - 1] == op ) {
            run++;
            k--;
        }
        if( run > 1 )
            o += (size_t) sprintf( out + o, "%zu", run );
        out[o++] = op;
    }
    out[o] = 0;
    free( ops );
    *cigar = out;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Driver (reference: src/algo/manager.c:120-185, searcher.c:155-174,       */
/* search_8.c:94-146, search_16.c:92-134, search_64.c:44-56,                */
/* db_adapter.c:212-239)                                                    */
/* ------------------------------------------------------------------------ */
int oracle_search( const oracle_config * cfg, const uint8_t * query, uint64_t qlen, uint64_t n_db,
        const uint8_t * db, const uint64_t * offsets, oracle_hit * out, uint64_t * out_len, oracle_stats * stats ) {
    heap hp;
    hp.alloc = cfg->hitcount;
    hp.count = 0;
    hp.a = malloc( (cfg->hitcount ? cfg->hitcount : 1) * sizeof(elem) );
    uint64_t cs = cfg->chunk_size ? cfg->chunk_size : 1000;
    seqlist chunk, o8, o16;
    chunk.ids = malloc( cs * sizeof(uint64_t) );
    chunk.seqs = malloc( cs * sizeof(uint8_t*) );
    chunk.lens = malloc( cs * sizeof(uint64_t) );
    o8.ids = malloc( cs * sizeof(uint64_t) );
    o8.seqs = malloc( cs * sizeof(uint8_t*) );
    o8.lens = malloc( cs * sizeof(uint64_t) );
    o16.ids = malloc( cs * sizeof(uint64_t) );
    o16.seqs = malloc( cs * sizeof(uint8_t*) );
    o16.lens = malloc( cs * sizeof(uint64_t) );
    pass_t p8, p16;
    pass_init( &p8, cfg, 8, cfg->lanes8, query, qlen );
    pass_init( &p16, cfg, 16, cfg->lanes16, query, qlen );
    stats->overflow8 = 0;
    stats->overflow16 = 0;

    for( uint64_t start = 0; start < n_db; start += cs ) {
        /* a chunk is an ID range; empty sequences are skipped (db_adapter.c:224-233) */
        chunk.n = 0;
        for( uint64_t id = start; id < start + cs && id < n_db; id++ ) {
            uint64_t len = offsets[id + 1] - offsets[id];
            if( len == 0 )
                continue;
            chunk.ids[chunk.n] = id;
            chunk.seqs[chunk.n] = db + offsets[id];
            chunk.lens[chunk.n] = len;
            chunk.n++;
        }
        /* a chunk without non-empty sequences ends the search: the reference's
         * search functions loop while( chunk->fill_pointer ) (search_8.c:652, search_16.c:785,
         * search_64.c:963), so later chunks are never read */
        if( chunk.n == 0 )
            break;
        const seqlist * to64 = NULL;
        if( cfg->bit_width == 64 ) {
            to64 = &chunk;
        }
        else if( cfg->bit_width == 16 ) {
            o16.n = 0;
            sink_t s = { &hp, &o16 };
            run_pass( &p16, &chunk, &s, NULL );
            stats->overflow16 += o16.n;
            to64 = &o16;
        }
        else {
            o8.n = 0;
            sink_t s8 = { &hp, &o8 };
            run_pass( &p8, &chunk, &s8, NULL );
            o16.n = 0;
            if( o8.n ) {
                stats->overflow8 += o8.n;
                sink_t s16 = { &hp, &o16 };
                run_pass( &p16, &o8, &s16, NULL );
                stats->overflow16 += o16.n;
            }
            to64 = &o16;
        }
        for( uint64_t k = 0; k < to64->n; k++ ) {
            int64_t sc = cfg->algo == 0 ? oracle_full_sw( cfg, to64->seqs[k], to64->lens[k], query, qlen )
                                        : oracle_full_nw( cfg, to64->seqs[k], to64->lens[k], query, qlen );
            heap_add( &hp, to64->ids[k], sc );
        }
    }
    qsort( hp.a, hp.count, sizeof(elem), elem_cmp );
    for( uint64_t h = 0; h < hp.count; h++ ) {
        oracle_hit * o = &out[h];
        memset( o, 0, sizeof(*o) );
        o->score = hp.a[h].score;
        o->id = hp.a[h].db_id;
        if( cfg->align_type == 1 ) {
            const uint8_t * d = db + offsets[o->id];
            uint64_t dl = offsets[o->id + 1] - offsets[o->id];
            oracle_align_pair( cfg, query, qlen, d, dl, &o->q_start, &o->q_end, &o->d_start, &o->d_end, &o->cigar );
        }
    }
    *out_len = hp.count;
    free( hp.a );
    free( chunk.ids );
    free( chunk.seqs );
    free( chunk.lens );
    free( o8.ids );
    free( o8.seqs );
    free( o8.lens );
    free( o16.ids );
    free( o16.seqs );
    free( o16.lens );
    return 0;
}

void oracle_free_hits( oracle_hit * hits, uint64_t n ) {
    for( uint64_t i = 0; i < n; i++ ) {
        free( hits[i].cigar );
        hits[i].cigar = NULL;
    }
}

/* ------------------------------------------------------------------------ */
/* Residue maps and matrices (reference: src/util/util_sequence.c:38-88,    */
/* src/query.c:102-130, src/util/util_sequence.c:298-318,                   */
/* src/matrices.c:388-460)                                                  */
/* ------------------------------------------------------------------------ */
static const char AA_SYMBOLS[] = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ";
static const char NT_SYMBOLS[] = "-ACMGRSVTWYHKDBN";

static int map_symbol( int c, int nucleotide ) {
    if( c >= 'a' && c <= 'z' )
        c = c - 'a' + 'A';
    if( nucleotide ) {
        if( c == 'U' )
            return 8; /* U reads as T */
        for( int k = 0; k < 16; k++ )
            if( NT_SYMBOLS[k] == c )
                return k;
        return -1;
    }
    if( c == '-' )
        return -1; /* code 0 has no symbol in the amino-acid map */
    for( int k = 1; k < 28; k++ )
        if( AA_SYMBOLS[k] == c )
            return k;
    return -1;
}

uint64_t oracle_map( const char * ascii, uint64_t n, int nucleotide, int drop_unknown, uint8_t * out ) {
    uint64_t o = 0;
    for( uint64_t i = 0; i < n; i++ ) {
        int m = map_symbol( (unsigned char) ascii[i], nucleotide );
        if( m >= 0 )
            out[o++] = (uint8_t) m;
        else if( !drop_unknown )
            out[o++] = 0;
    }
    return o;
}

void oracle_constant_matrix( int match, int mismatch, int64_t * out ) {
    for( int k = 0; k < 1024; k++ )
        out[k] = -1;
    for( int a = 1; a < 32; a++ )
        for( int b = 1; b < 32; b++ )
            out[(a << 5) + b] = (int8_t) (a == b ? match : mismatch);
}

int oracle_parse_matrix( const char * text, int64_t * out ) {
    for( int k = 0; k < 1024; k++ )
        out[k] = -1;
    int order[256];
    int symbols = 0;
    const char * s = text;
    while( *s ) {
        const char * e = strchr( s, '\n' );
        size_t n = e ? (size_t) (e - s) : strlen( s );
        char line[4096];
        if( n >= sizeof(line) )
            n = sizeof(line) - 1;
        memcpy( line, s, n );
        line[n] = 0;
        s = e ? e + 1 : s + strlen( s );
        char c = line[0];
        if( c == 0 || c == '#' )
            continue;
        if( c == ' ' || c == '\t' ) {
            /* header: the column symbols (matrices.c:399-410) */
            for( char * p = line + 1; *p; p++ )
                if( *p != ' ' && *p != '\t' && *p != '\n' && symbols < 256 )
                    order[symbols++] = map_symbol( (unsigned char) *p, 0 );
            continue;
        }
        int a = map_symbol( (unsigned char) c, 0 );
        char * p = line + 1;
        for( int i = 0; i < symbols; i++ ) {
            char * end;
            long v = strtol( p, &end, 10 );
            if( end == p )
                return -1;
            p = end;
            int b = order[i];
            if( a >= 0 && b >= 0 )
                out[(a << 5) + b] = v;
        }
    }
    return 0;
}
