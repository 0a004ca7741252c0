// api.cpp -- the libssa.h entry points of the B200 build.
//
// The public functions keep the reference's names, argument meaning, global
// state, messages and error behaviour (reference: src/libssa.c:38-271,
// src/query.c, src/matrices.c, src/util/util.c:36-98).  Configuration errors
// print to stderr and exit(1) like the reference's fatal(); a bad query file
// prints an error and returns NULL.  The search itself is delegated to the
// GPU engine (engine.cu); there is no CPU search path.
#include "ssa_internal.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include "libssa_b200.h"
#include "libssa_extern_db.h"

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <strings.h>

namespace ssa {

Config & config() {
    static Config c;
    return c;
}

// ---- messages (reference: src/util/util.c:36-89) -------------------------------
void fatal( const char * fmt, ... ) {
    if( fmt ) {
        va_list ap;
        va_start( ap, fmt );
        vfprintf( stderr, fmt, ap );
        fprintf( stderr, "\n" );
        va_end( ap );
    }
    exit( 1 );
}

static void emit( int level, const char * prefix, bool newline, const char * fmt, va_list ap ) {
    if( level > config().output_mode )
        return;
    printf( "%s", prefix );
    vprintf( fmt, ap );
    if( newline )
        printf( "\n" );
}

void print_info( const char * fmt, ... ) {
    va_list ap;
    va_start( ap, fmt );
    emit( OUTPUT_INFO, "libssa INFO: ", false, fmt, ap );
    va_end( ap );
}

void print_warning( const char * fmt, ... ) {
    va_list ap;
    va_start( ap, fmt );
    emit( OUTPUT_WARNING, "libssa WARNING: ", true, fmt, ap );
    va_end( ap );
}

void print_error( const char * fmt, ... ) {
    va_list ap;
    va_start( ap, fmt );
    emit( OUTPUT_ERROR, "libssa ERROR: ", true, fmt, ap );
    va_end( ap );
}

// ---- residue maps (reference: src/util/util_sequence.c:38-88) ------------------
// Code k of the amino-acid alphabet is AA_SYMBOLS[k] (code 0, the pad, has no
// symbol); nucleotides use the IUPAC nt16 bit codes with U read as T.
static const char AA_SYMBOLS[] = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ";
static const char NT_SYMBOLS[] = "-ACMGRSVTWYHKDBN";

struct Maps {
    signed char aa[256];
    signed char nt[256];
    Maps() {
        memset( aa, -1, sizeof(aa) );
        memset( nt, -1, sizeof(nt) );
        for( int k = 1; k < 28; k++ ) {
            unsigned char c = (unsigned char) AA_SYMBOLS[k];
            aa[c] = (signed char) k;
            if( c >= 'A' && c <= 'Z' )
                aa[c - 'A' + 'a'] = (signed char) k;
        }
        for( int k = 0; k < 16; k++ ) {
            unsigned char c = (unsigned char) NT_SYMBOLS[k];
            nt[c] = (signed char) k;
            if( c >= 'A' && c <= 'Z' )
                nt[c - 'A' + 'a'] = (signed char) k;
        }
        nt[(unsigned char) 'U'] = nt[(unsigned char) 'T'];
        nt[(unsigned char) 'u'] = nt[(unsigned char) 'T'];
    }
};

static const Maps & maps() {
    static Maps m;
    return m;
}

int map_aa( unsigned char c ) {
    return maps().aa[c];
}

int map_nt16( unsigned char c ) {
    return maps().nt[c];
}

// ---- matrices (reference: src/matrices.c:335-568) ------------------------------
struct BuiltinMatrix {
    const char * name;
    const char * symbols;
    int values[25 * 25];
};

static const BuiltinMatrix BUILTINS[] = {
#include "builtin_matrices.inc"
};

static void matrix_clear( int64_t * out ) {
    for( int k = 0; k < 1024; k++ )
        out[k] = -1;   // unset cells score -1 (reference: src/matrices.c:344)
}

bool matrix_builtin( const char * name, int64_t * out ) {
    for( const BuiltinMatrix & m : BUILTINS ) {
        if( strcasecmp( name, m.name ) != 0 )
            continue;
        matrix_clear( out );
        const int n = (int) strlen( m.symbols );
        for( int a = 0; a < n; a++ ) {
            int ca = map_aa( (unsigned char) m.symbols[a] );
            for( int b = 0; b < n; b++ ) {
                int cb = map_aa( (unsigned char) m.symbols[b] );
                if( ca >= 0 && cb >= 0 )
                    out[(ca << 5) + cb] = m.values[a * n + b];
            }
        }
        return true;
    }
    return false;
}

// Matrix text: '#' comments and blank lines are skipped, a line starting
// with blank space lists the column symbols, every other line is a row symbol
// followed by one score per column symbol (reference: src/matrices.c:388-437).
void matrix_from_string( const char * text, int64_t * out ) {
    matrix_clear( out );
    std::vector<int> order;
    const char * s = text;
    while( *s ) {
        const char * e = strchr( s, '\n' );
        const size_t n = e ? (size_t) (e - s) : strlen( s );
        std::string line( s, n );
        s = e ? e + 1 : s + n;
        if( line.empty() || line[0] == '#' )
            continue;
        if( line[0] == ' ' || line[0] == '\t' ) {
            for( size_t k = 1; k < line.size(); k++ )
                if( !strchr( " \t\n\r", line[k] ) )
                    order.push_back( map_aa( (unsigned char) line[k] ) );
            continue;
        }
        const int a = map_aa( (unsigned char) line[0] );
        const char * p = line.c_str() + 1;
        for( size_t i = 0; i < order.size(); i++ ) {
            char * end;
            long v = strtol( p, &end, 10 );
            if( end == p )
                fatal( "Problem parsing score matrix file." );
            p = end;
            const int b = order[i];
            if( a >= 0 && b >= 0 )
                out[(a << 5) + b] = v;
        }
    }
}

void matrix_constant( int match, int mismatch, int64_t * out ) {
    // reference: src/matrices.c:447-460 -- code 0 keeps -1
    matrix_clear( out );
    for( int a = 1; a < 32; a++ )
        for( int b = 1; b < 32; b++ )
            out[(a << 5) + b] = (int8_t) (a == b ? match : mismatch);
}

// ---- genetic codes and translation (reference: src/util/util_sequence.c:88-260,
//      298-392) ----------------------------------------------------------------------
// NCBI translation tables 1-25, one amino acid per codon with the codons in
// TCAG order (TTT, TTC, TTA, TTG, TCT, ...); tables 7, 8 and 17-20 do not exist.
static const char * const NCBI_CODES[25] = {
    "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIMMTTTTNNKKSS**VVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWTTTTPPPPHHQQRRRRIIMMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIMMTTTTNNKKSSSSVVVVAAAADDEEGGGG",
    "FFLLSSSSYYQQCC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    nullptr,
    nullptr,
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIIMTTTTNNNKSSSSVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCCWLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CC*WLLLSPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIMMTTTTNNKKSSGGVVVVAAAADDEEGGGG",
    "FFLLSSSSYYY*CCWWLLLLPPPPHHQQRRRRIIIMTTTTNNNKSSSSVVVVAAAADDEEGGGG",
    "FFLLSSSSYY*QCC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY*LCC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    nullptr,
    nullptr,
    nullptr,
    nullptr,
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIMMTTTTNNNKSSSSVVVVAAAADDEEGGGG",
    "FFLLSS*SYY*LCC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FF*LSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCWWLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSSKVVVVAAAADDEEGGGG",
    "FFLLSSSSYY**CCGWLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG",
};

// Amino-acid code of every triple (a, b, c) of nt16 codes (bit 0 A, 1 C, 2 G,
// 3 T): the amino acid all concrete codons the IUPAC codes allow agree on, B
// when they give D and N, Z when they give E and Q, X otherwise (and for a
// code without bases).
void translation_table( int code_no, uint8_t * table ) {
    static const int tcag[4] = { 2, 1, 3, 0 };   // base bit -> TCAG position
    const char * code = (code_no >= 1 && code_no <= 25) ? NCBI_CODES[code_no - 1] : nullptr;
    if( !code )
        fatal( "Illegal genetic code %d.", code_no );
    for( int t = 0; t < 4096; t++ ) {
        const int m[3] = { t >> 8, (t >> 4) & 15, t & 15 };
        bool seen[128] = {};
        int n = 0;
        char one = 'X';
        for( int i = 0; i < 4; i++ )
            for( int j = 0; j < 4; j++ )
                for( int k = 0; k < 4; k++ ) {
                    if( !((m[0] >> i) & 1) || !((m[1] >> j) & 1) || !((m[2] >> k) & 1) )
                        continue;
                    const char x = code[tcag[i] * 16 + tcag[j] * 4 + tcag[k]];
                    if( !seen[(int) x] ) {
                        seen[(int) x] = true;
                        n++;
                        one = x;
                    }
                }
        char aa = 'X';
        if( n == 1 )
            aa = one;
        else if( n == 2 && seen['D'] && seen['N'] )
            aa = 'B';
        else if( n == 2 && seen['E'] && seen['Q'] )
            aa = 'Z';
        table[t] = (uint8_t) map_aa( (unsigned char) aa );
    }
}

uint32_t units_per_record( int symtype, int strands ) {
    return (symtype == NUCLEOTIDE && (strands & 2)) ? 2u : 1u;
}

// complement of an nt16 code: A <-> T, C <-> G bit by bit
uint8_t nt_complement( uint8_t x ) {
    return (uint8_t) (((x & 1) << 3) | ((x & 2) << 1) | ((x & 4) >> 1) | ((x & 8) >> 3));
}

// Protein of one strand (0 forward, 1 reverse complement) and frame (0-2) of a
// mapped nucleotide sequence: codon k starts at frame + 3k on that strand.
void translate( const char * dna, size_t n, int strand, int frame, const uint8_t * table, std::vector<char> & out ) {
    const size_t len = (n > (size_t) frame) ? (n - frame) / 3 : 0;
    out.assign( len + 1, 0 );
    for( size_t k = 0; k < len; k++ ) {
        int c;
        if( strand == 0 ) {
            const size_t p = frame + 3 * k;
            c = (dna[p] << 8) | (dna[p + 1] << 4) | dna[p + 2];
        }
        else {
            const size_t p = n - 1 - frame - 3 * k;
            c = (nt_complement( (uint8_t) dna[p] ) << 8) | (nt_complement( (uint8_t) dna[p - 1] ) << 4) |
                    nt_complement( (uint8_t) dna[p - 2] );
        }
        out[k] = (char) table[c & 4095];
    }
}

}  // namespace ssa

using namespace ssa;

// ---- the query object ------------------------------------------------------------
// One sequence a search runs for the query: the mapped residues themselves, a
// strand of a nucleotide query, or a translated frame (reference:
// src/query.c:132-160, src/algo/searcher.c:58-85).
struct QueryFrame {
    std::vector<char> seq;   // codes, NUL-terminated
    int strand;
    int frame;
};

struct _query {
    char * seq;          // mapped codes, NUL-terminated
    size_t len;
    char * header;
    size_t headerlen;
    int symtype;         // symbol type the codes were mapped with
    std::vector<QueryFrame> * frames;   // sequences searched, in the reference's query order
};

// Strands of a nucleotide query, or translated frames, as the settings at read
// time ask for; otherwise the mapped sequence alone.
static void make_frames( p_query q ) {
    const Config & c = config();
    q->frames = new std::vector<QueryFrame>();
    if( c.symtype == NUCLEOTIDE ) {
        if( c.strands & 1 )
            q->frames->push_back( QueryFrame{ std::vector<char>( q->seq, q->seq + q->len + 1 ), 0, 0 } );
        if( c.strands & 2 ) {
            std::vector<char> rc( q->len + 1, 0 );
            for( size_t i = 0; i < q->len; i++ )
                rc[i] = (char) nt_complement( (uint8_t) q->seq[q->len - 1 - i] );
            q->frames->push_back( QueryFrame{ std::move( rc ), 1, 0 } );
        }
    }
    else if( c.symtype == TRANS_QUERY || c.symtype == TRANS_BOTH ) {
        uint8_t table[4096];
        translation_table( c.q_gencode, table );
        for( int st = 0; st < 2; st++ ) {
            if( !((st + 1) & c.strands) )
                continue;
            for( int f = 0; f < 3; f++ ) {
                QueryFrame qf{ {}, st, f };
                translate( q->seq, q->len, st, f, table, qf.seq );
                q->frames->push_back( std::move( qf ) );
            }
        }
    }
    else {
        q->frames->push_back( QueryFrame{ std::vector<char>( q->seq, q->seq + q->len + 1 ), 0, 0 } );
    }
}

static bool nucleotide_map( int symtype ) {
    return !(symtype == AMINOACID || symtype == TRANS_DB);
}

// Maps ASCII to codes, removing unknown symbols with a warning; whitespace is
// dropped silently (reference: src/query.c:102-130).
static p_query make_query( const char * text, size_t n, char * header, size_t headerlen ) {
    const bool nt = nucleotide_map( config().symtype );
    p_query q = (p_query) calloc( 1, sizeof(struct _query) );
    q->seq = (char *) malloc( n + 1 );
    std::string unknown;
    size_t k = 0;
    for( size_t i = 0; i < n; i++ ) {
        const unsigned char c = (unsigned char) text[i];
        const int m = nt ? map_nt16( c ) : map_aa( c );
        if( m >= 0 )
            q->seq[k++] = (char) m;
        else if( c != '\n' && c != ' ' && c != '\t' )
            unknown += (char) c;
    }
    if( !unknown.empty() )
        print_warning( "%zu unknown symbols found and removed: '%s'", unknown.size(), unknown.c_str() );
    q->seq[k] = 0;
    q->len = k;
    q->header = header;
    q->headerlen = headerlen;
    q->symtype = config().symtype;
    make_frames( q );
    return q;
}

static p_query query_from_file( const char * filename ) {
    // reference: src/query.c:187-264
    if( strcmp( filename, "-" ) == 0 ) {
        print_error( "Query not specified" );
        return nullptr;
    }
    FILE * fp = fopen( filename, "r" );
    if( !fp ) {
        print_error( "Cannot open query file: %s", filename );
        return nullptr;
    }
    char line[2048];
    line[0] = 0;
    if( !fgets( line, sizeof(line), fp ) ) {
        print_error( "Could not initialise from query sequence" );
        fclose( fp );
        return nullptr;
    }
    size_t len = strlen( line );
    if( len && line[len - 1] == '\n' ) {
        line[len - 1] = 0;
        len--;
    }
    char * header = nullptr;
    size_t headerlen = 0;
    if( line[0] == '>' ) {
        header = (char *) malloc( len + 1 );
        memcpy( header, line + 1, len );
        header[len] = 0;
        headerlen = len ? len - 1 : 0;
        line[0] = 0;
        if( !fgets( line, sizeof(line), fp ) ) {
            print_error( "Could not read first line from query sequence" );
            free( header );
            fclose( fp );
            return nullptr;
        }
    }
    std::string seq;
    while( line[0] && line[0] != '>' ) {
        seq += line;
        if( !fgets( line, sizeof(line), fp ) )
            break;
    }
    fclose( fp );
    return make_query( seq.data(), seq.size(), header, headerlen );
}

// ---- alignment lists -----------------------------------------------------------
static p_alignment_list make_list( const std::vector<Hit> & hits, p_query q, bool with_cigar ) {
    p_alignment_list l = (p_alignment_list) malloc( sizeof(alignment_list_t) );
    l->len = hits.size();
    l->alignments = (p_alignment *) malloc( std::max<size_t>( 1, hits.size() ) * sizeof(p_alignment) );
    const bool nt = config().symtype == NUCLEOTIDE;
    for( size_t k = 0; k < hits.size(); k++ ) {
        const Hit & h = hits[k];
        p_alignment a = (p_alignment) calloc( 1, sizeof(alignment_t) );
        // the hit's database record is fetched and mapped again, as the
        // reference does per hit (reference: src/algo/aligner.c:62-93); a
        // reverse-complement unit is mapped forward there too (us_prepare_sequence
        // only reverses for strand 2, which the database units never carry)
        p_seqinfo info = ssa_db_get_sequence( h.id );
        if( !info )
            fatal( "Could not get sequence from DB: %u", h.id );
        const QueryFrame & qf = (*q->frames)[h.q_index];
        a->db_seq.seq = (char *) malloc( info->seqlen + 1 );
        for( size_t i = 0; i < info->seqlen; i++ ) {
            int m = nt ? map_nt16( (unsigned char) info->seq[i] ) : map_aa( (unsigned char) info->seq[i] );
            a->db_seq.seq[i] = (char) (m < 0 ? 0 : m);
        }
        a->db_seq.seq[info->seqlen] = 0;
        a->db_seq.len = info->seqlen;
        a->db_seq.ID = info->ID;
        // the reference stores the unit's frame in strand and its strand in
        // frame (reference: src/algo/aligner.c:76-77)
        a->db_seq.strand = h.db_frame;
        a->db_seq.frame = h.db_strand;
        a->query.seq = const_cast<char *>( qf.seq.data() );
        a->query.len = qf.seq.size() - 1;
        a->query.strand = qf.strand;
        a->query.frame = qf.frame;
        a->score = (long) h.score;
        if( with_cigar && h.has_cigar ) {
            a->alignment = (char *) malloc( h.cigar.size() + 1 );
            memcpy( a->alignment, h.cigar.c_str(), h.cigar.size() + 1 );
            a->alignment_len = h.cigar.size();
            a->align_q_start = h.q_start;
            a->align_q_end = h.q_end;
            a->align_d_start = h.d_start;
            a->align_d_end = h.d_end;
        }
        l->alignments[k] = a;
    }
    return l;
}

static SearchStats g_last_stats;

// Checks shared by sw_align/nw_align (reference: src/libssa.c:196-219).
static void test_configuration( p_query query ) {
    const Config & c = config();
    if( !c.gap_open && !c.gap_extend )
        print_warning( "Gap opening and gap extension cost set to zero. Possible error." );
    if( !c.matrix_set )
        fatal( "Scoring not initialized." );
    if( !query )
        fatal( "Query not initialized." );
    if( ssa_db_get_sequence_count() == 0 )
        print_warning( "Database contains zero sequences. Possible error." );
    if( !c.constant_scoring && c.symtype == NUCLEOTIDE )
        fatal( "Nucleotide sequences can only be aligned using constant scores." );
}

static SearchRequest make_request( int algo, size_t hitcount, int bit_width, int align_type ) {
    const Config & c = config();
    if( bit_width != BIT_WIDTH_8 && bit_width != BIT_WIDTH_16 && bit_width != BIT_WIDTH_64 )
        fatal( "\nunknown bit width provided: %d\n\n", bit_width );
    // the reference crashes (segmentation fault) in the searches of a
    // translated database, so there is no behaviour to reproduce
    if( c.symtype == TRANS_DB || c.symtype == TRANS_BOTH )
        fatal( "Searches of a translated database (symbol type %d) are not supported by the B200 build.",
                c.symtype );
    if( c.symtype != AMINOACID && c.symtype != NUCLEOTIDE && c.symtype != TRANS_QUERY )
        fatal( "Illegal symbol type specified." );
    SearchRequest r;
    r.algo = algo;
    r.bit_width = bit_width;
    r.align_type = align_type;
    r.hitcount = hitcount;
    r.chunk_size = c.chunk_size;
    // lane counts of the CPU schedule whose hit order is reproduced
    // (reference: src/cpu_config.c:29-33, src/algo/8/search_8.c:41-56)
    if( c.simd_mode >= COMPUTE_ON_AVX2 ) {
        r.lanes8 = 32;
        r.lanes16 = 16;
    }
    else if( c.simd_mode == COMPUTE_ON_SSE41 ) {
        r.lanes8 = 16;
        r.lanes16 = 8;
    }
    else {
        if( bit_width == BIT_WIDTH_8 )
            fatal( "\nAVX2 and SSE4.1 not enabled. No 8 bit search possible\n\n" );
        r.lanes8 = 16;
        r.lanes16 = 8;
    }
    r.gap_open = c.gap_open;
    r.gap_extend = c.gap_extend;
    r.matrix = c.matrix;
    return r;
}

static std::vector<p_alignment_list> run_search( int algo, p_query * queries, size_t n, size_t hitcount,
        int bit_width, int align_type ) {
    for( size_t i = 0; i < n; i++ )
        test_configuration( queries[i] );
    SearchRequest req = make_request( algo, hitcount, bit_width, align_type );
    // every strand or frame of a query is searched as its own sequence; the
    // engine merges a query's frames into one heap as the reference does
    std::vector<QueryCodes> qc;
    std::vector<uint32_t> groups( n );
    for( size_t i = 0; i < n; i++ ) {
        if( queries[i]->symtype != config().symtype )
            fatal( "Query was read with a different symbol type than the current one." );
        if( queries[i]->len == 0 )
            fatal( "Query sequence is empty." );
        for( const QueryFrame & f : *queries[i]->frames ) {
            if( f.seq.size() <= 1 )
                fatal( "Query frame (strand %d, frame %d) is empty.", f.strand, f.frame );
            qc.push_back( QueryCodes{ (const uint8_t *) f.seq.data(), (uint32_t) (f.seq.size() - 1) } );
        }
        groups[i] = (uint32_t) queries[i]->frames->size();
    }
    std::vector<std::vector<Hit>> hits;
    SearchStats st;
    engine_search( req, qc, groups, hits, st );
    if( st.overflow8 || st.overflow16 )
        print_info( "Overflow occurred: %ld sequences were re-aligned with 16 bit, and %ld sequences with 64 bit\n",
                (long) st.overflow8, (long) st.overflow16 );
    g_last_stats = st;
    std::vector<p_alignment_list> out( n );
    for( size_t i = 0; i < n; i++ )
        out[i] = make_list( hits[i], queries[i], align_type == COMPUTE_ALIGNMENT );
    return out;
}

// ---- serving ------------------------------------------------------------------------
// A server owns a fixed set of query slots resident on the device.  Its loop
// thread repeats waves: admit waiting requests into free slots (first come,
// first served, while their traceback memory fits the budget), run the entry
// pass and cascade of every occupied slot over the next segment of the
// database (the segments form a ring, so a request admitted at any wave starts
// with the segment the loop is on and is done after one full turn), then finish
// the requests that have seen every segment: replay of the CPU lane schedule,
// heap, traceback, alignment list.  Per (query, sequence) the work is the same
// as in sw_align/nw_align, so every result equals the one the query gets alone.
struct ServeTicket {
    p_query query = nullptr;
    long long id = 0;
    uint64_t mem = 0;
    int slot = -1;
    uint32_t waves = 0;
    bool done = false;
    bool waited = false;       // left waiting at an admission point (no free slot or memory)
    std::chrono::steady_clock::time_point t_submit, t_done;
    ReplayQuery lists;
    p_alignment_list result = nullptr;
};

struct ServerImpl {
    SearchRequest req;
    std::vector<int64_t> matrix;       // the settings at start, kept for the server's lifetime
    uint32_t slots = 0;
    std::vector<uint32_t> seg;         // segment bounds over the length-sorted sequences
    uint64_t budget = 0;
    uint64_t max_db_len = 0;
    uint64_t residues = 0;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<ServeTicket *> pending;
    std::map<long long, ServeTicket *> tickets;
    std::vector<ServeTicket *> owner;  // per slot
    uint32_t occupied = 0;
    uint64_t mem_in_use = 0;
    long long next_id = 0;
    bool stopping = false;
    uint32_t cursor = 0;
    std::thread loop_thread;
    // statistics
    uint64_t submitted = 0, completed = 0, waves = 0, cells = 0;
    uint64_t queued = 0, slot_waves = 0;
    uint32_t max_pending = 0, max_occupied = 0;
    double busy_seconds = 0, device_seconds = 0;

    void loop();
};

void ServerImpl::loop() {
    const uint32_t n_seg = (uint32_t) seg.size() - 1;
    for( ;; ) {
        std::vector<ServeTicket *> admitted;
        {
            std::unique_lock<std::mutex> lk( m );
            cv_work.wait( lk, [&] { return stopping || !pending.empty() || occupied > 0; } );
            if( pending.empty() && occupied == 0 )
                break;     // stopping and drained
            while( !pending.empty() && occupied < slots ) {
                ServeTicket * t = pending.front();
                if( budget && occupied > 0 && mem_in_use + t->mem > budget )
                    break;
                pending.pop_front();
                uint32_t s = 0;
                while( owner[s] )
                    s++;
                owner[s] = t;
                t->slot = (int) s;
                occupied++;
                mem_in_use += t->mem;
                admitted.push_back( t );
            }
            // requests this admission point could not take wait for a later wave
            for( ServeTicket * t : pending ) {
                if( !t->waited ) {
                    t->waited = true;
                    queued++;
                }
            }
            max_pending = std::max<uint32_t>( max_pending, (uint32_t) pending.size() );
            max_occupied = std::max( max_occupied, occupied );
            slot_waves += occupied;
        }
        const auto t0 = std::chrono::steady_clock::now();
        for( ServeTicket * t : admitted )
            engine_serve_load( (uint32_t) t->slot, (const uint8_t *) t->query->seq, (uint32_t) t->query->len );
        std::vector<uint32_t> active;
        for( uint32_t s = 0; s < slots; s++ )
            if( owner[s] )
                active.push_back( s );
        std::vector<ServeOverflow> oe, o16;
        SearchStats st;
        engine_serve_wave( req, active, seg[cursor], seg[cursor + 1], oe, o16, st );
        cursor = (cursor + 1) % n_seg;
        for( const ServeOverflow & o : oe )
            owner[o.slot]->lists.ovf_entry.emplace_back( o.id, o.nb );
        for( const ServeOverflow & o : o16 )
            owner[o.slot]->lists.ovf16.emplace_back( o.id, o.nb );
        std::vector<uint32_t> done;
        std::vector<ReplayQuery> rq;
        for( uint32_t s : active ) {
            ServeTicket * t = owner[s];
            if( ++t->waves == n_seg ) {
                done.push_back( s );
                rq.push_back( std::move( t->lists ) );
            }
        }
        std::vector<std::vector<Hit>> hits;
        if( !done.empty() )
            engine_serve_finish( req, done, rq, hits, st );
        std::vector<p_alignment_list> lists( done.size() );
        for( size_t i = 0; i < done.size(); i++ )
            lists[i] = make_list( hits[done[i]], owner[done[i]]->query, req.align_type == COMPUTE_ALIGNMENT );
        const auto t1 = std::chrono::steady_clock::now();
        {
            std::lock_guard<std::mutex> lk( m );
            waves++;
            busy_seconds += std::chrono::duration<double>( t1 - t0 ).count();
            device_seconds += st.kernel_seconds;
            for( size_t i = 0; i < done.size(); i++ ) {
                ServeTicket * t = owner[done[i]];
                t->result = lists[i];
                t->done = true;
                t->t_done = t1;
                cells += (uint64_t) t->query->len * residues;
                completed++;
                mem_in_use -= t->mem;
                owner[done[i]] = nullptr;
                occupied--;
            }
        }
        if( !done.empty() )
            cv_done.notify_all();
    }
}

// ---- libssa.h ---------------------------------------------------------------------
// The C entry points are the library's only exported symbols.
#pragma GCC visibility push( default )
extern "C" {

void set_output_mode( int mode ) {
    config().output_mode = mode;
}

void set_simd_compute_mode( int mode ) {
    config().simd_mode = mode;
}

void set_chunk_size( size_t size ) {
    if( size == 0 ) {
        print_error( "Only non zero chunk sizes are allowed. Using the default size of 1000 sequences.", size );
        size = 1000;
    }
    config().chunk_size = size;
}

void set_thread_count( size_t count ) {
    config().thread_count = count;
}

void init_score_matrix( int mode, const char * matrix ) {
    Config & c = config();
    if( mode == READ_FROM_FILE ) {
        FILE * fp = fopen( matrix, "r" );
        if( !fp )
            fatal( "Cannot open score matrix file." );
        std::string text;
        char buf[4096];
        size_t n;
        while( (n = fread( buf, 1, sizeof(buf), fp )) > 0 )
            text.append( buf, n );
        fclose( fp );
        matrix_from_string( text.c_str(), c.matrix );
    }
    else if( mode == READ_FROM_STRING ) {
        if( !matrix )
            fatal( "Cannot read score matrix string." );
        matrix_from_string( matrix, c.matrix );
    }
    else if( mode == MATRIX_BUILDIN ) {
        if( !matrix_builtin( matrix, c.matrix ) )
            fatal( "Unknown matrix: %s", matrix );
    }
    else {
        fatal( "Unknown mode for reading score matrices: %d", mode );
    }
    c.matrix_set = true;
    c.constant_scoring = false;
}

void init_constant_scores( const int8_t p, const int8_t m ) {
    Config & c = config();
    matrix_constant( p, m, c.matrix );
    c.matrix_set = true;
    c.constant_scoring = true;
}

void init_gap_penalties( const int8_t gapO, const int8_t gapE ) {
    config().gap_open = gapO;
    config().gap_extend = gapE;
}

void init_symbol_translation( int type, int strands, int db_gencode, int q_gencode ) {
    // reference: src/libssa.c:139-157 (the range checks read the previous
    // symbol type, as there)
    static const bool known[24] = { false, true, true, true, true, true, true, false, false, true, true, true, true,
        true, true, true, true, false, false, false, false, true, true, true };
    Config & c = config();
    if( q_gencode < 1 || q_gencode > 23 || !known[q_gencode] )
        fatal( "Illegal query genetic code specified." );
    if( db_gencode < 1 || db_gencode > 23 || !known[db_gencode] )
        fatal( "Illegal database genetic code specified." );
    if( c.symtype < 0 || c.symtype > 4 )
        fatal( "Illegal symbol type specified." );
    if( c.symtype < 0 || c.symtype > 2 )
        fatal( "Illegal strands specified." );
    c.symtype = type;
    c.strands = strands;
    c.db_gencode = db_gencode;
    c.q_gencode = q_gencode;
}

void init_db( const char * db_file ) {
    ssa_db_close();
    ssa_db_init( db_file );
    engine_invalidate_database();
    print_info( "DB read %lu sequences\n", (unsigned long) ssa_db_get_sequence_count() );
}

p_query init_sequence_fasta( int mode, const char * fasta ) {
    if( mode == READ_FROM_FILE )
        return query_from_file( fasta );
    if( mode == READ_FROM_STRING )
        return make_query( fasta, strlen( fasta ), nullptr, 0 );
    fatal( "Unknown mode for reading query sequences: %d", mode );
}

void free_sequence( p_query p ) {
    if( !p )
        return;
    free( p->seq );
    free( p->header );
    delete p->frames;
    free( p );
}

p_alignment_list sw_align( p_query p, size_t hitcount, int bit_width, int align_type ) {
    return run_search( 0, &p, 1, hitcount, bit_width, align_type )[0];
}

p_alignment_list nw_align( p_query p, size_t hitcount, int bit_width, int align_type ) {
    return run_search( 1, &p, 1, hitcount, bit_width, align_type )[0];
}

void free_alignment( p_alignment_list alist ) {
    if( !alist )
        return;
    for( size_t i = 0; i < alist->len; i++ ) {
        p_alignment a = alist->alignments[i];
        if( !a )
            continue;
        free( a->db_seq.seq );
        free( a->alignment );
        free( a );
    }
    free( alist->alignments );
    free( alist );
}

void ssa_exit( void ) {
    config().matrix_set = false;
    ssa_db_close();
    engine_shutdown();
}

// ---- libssa_b200.h extensions -------------------------------------------------------
int ssa_align_batch( int algorithm, p_query * queries, size_t n_queries, size_t hitcount, int bit_width,
        int align_type, p_alignment_list * results ) {
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH )
        fatal( "\nUnknown search type: %d\n\n", algorithm );
    if( n_queries == 0 )
        return 0;
    if( !queries || !results )
        fatal( "Query not initialized." );
    std::vector<p_alignment_list> l =
            run_search( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, queries, n_queries, hitcount, bit_width, align_type );
    for( size_t i = 0; i < n_queries; i++ )
        results[i] = l[i];
    return 0;
}

// Long pairs: queries[i] against database sequence db_ids[i] alone.  The
// reference's equivalent is init_db of that one sequence and
// sw_align / nw_align( queries[i], 1, bit_width, align_type ) per pair; every
// entry width of the reference reports the exact score there (a saturated lane
// is searched again at the next width), which is what the pair kernel computes,
// provided the narrow lanes hold the score table and gap costs untruncated.
int ssa_align_pairs( int algorithm, p_query * queries, const size_t * db_ids, size_t n_pairs, int bit_width,
        int align_type, p_alignment_list * results ) {
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH )
        fatal( "\nUnknown search type: %d\n\n", algorithm );
    if( n_pairs == 0 )
        return 0;
    if( !queries || !db_ids || !results )
        fatal( "Query not initialized." );
    for( size_t i = 0; i < n_pairs; i++ )
        test_configuration( queries[i] );
    const Config & c = config();
    SearchRequest req = make_request( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, 1, bit_width, align_type );
    if( c.symtype == TRANS_QUERY || (c.symtype == NUCLEOTIDE && c.strands != FORWARD_STRAND) ) {
        print_error( "ssa_align_pairs: translated or two-strand searches are not supported" );
        return -1;
    }
    if( c.gap_open > 0 || c.gap_extend > 0 ) {
        print_error( "ssa_align_pairs: positive gap costs are not supported" );
        return -1;
    }
    const int64_t lo = bit_width == BIT_WIDTH_8 ? INT8_MIN : bit_width == BIT_WIDTH_16 ? INT16_MIN : INT64_MIN;
    const int64_t hi = bit_width == BIT_WIDTH_8 ? INT8_MAX : bit_width == BIT_WIDTH_16 ? INT16_MAX : INT64_MAX;
    bool fits = (int64_t) c.gap_open + c.gap_extend >= lo;
    for( int k = 0; k < 1024; k++ )
        fits = fits && c.matrix[k] >= lo && c.matrix[k] <= hi;
    if( !fits ) {
        print_error( "ssa_align_pairs: the score matrix or the gap costs do not fit the %d-bit entry width", bit_width );
        return -1;
    }
    const HostDb & db = engine_database();
    if( db.upi != 1 ) {
        print_error( "ssa_align_pairs: translated or two-strand searches are not supported" );
        return -1;
    }
    std::vector<QueryCodes> qc( n_pairs );
    std::vector<uint32_t> units( n_pairs );
    for( size_t i = 0; i < n_pairs; i++ ) {
        if( queries[i]->symtype != c.symtype )
            fatal( "Query was read with a different symbol type than the current one." );
        if( queries[i]->len == 0 )
            fatal( "Query sequence is empty." );
        const QueryFrame & f = (*queries[i]->frames)[0];
        qc[i] = QueryCodes{ (const uint8_t *) f.seq.data(), (uint32_t) (f.seq.size() - 1) };
        if( db_ids[i] >= db.n_records ) {
            print_error( "ssa_align_pairs: database ID %zu out of range (%zu sequences)", db_ids[i],
                    (size_t) db.n_records );
            return -1;
        }
        units[i] = (uint32_t) db_ids[i];
    }
    std::vector<std::vector<Hit>> hits;
    SearchStats st;
    engine_align_pairs( req, qc, units, hits, st );
    g_last_stats = st;
    for( size_t i = 0; i < n_pairs; i++ )
        results[i] = make_list( hits[i], queries[i], align_type == COMPUTE_ALIGNMENT );
    return 0;
}

void ssa_b200_set_traceback_memory( size_t bytes ) {
    engine_set_traceback_memory( (uint64_t) bytes );
}

void ssa_b200_set_db_memory( size_t bytes ) {
    engine_set_db_memory( (uint64_t) bytes );
}

int ssa_b200_db_streamed( void ) {
    return engine_streaming() ? 1 : 0;
}

void ssa_get_stats( ssa_stats_t * out ) {
    if( !out )
        return;
    out->overflow_8_to_16 = g_last_stats.overflow8;
    out->overflow_16_to_64 = g_last_stats.overflow16;
    out->cells = g_last_stats.cells;
    out->gpu_seconds = g_last_stats.seconds_gpu;
    out->kernel_launches_total = engine_kernel_launches();
    out->entry_seconds = g_last_stats.entry_seconds;
    out->kernel_seconds = g_last_stats.kernel_seconds;
    out->h2d_bytes = g_last_stats.h2d_bytes;
    out->d2h_bytes = g_last_stats.d2h_bytes;
}

// ---- database-sharded searches ----------------------------------------------------
// Shared checks: one query sequence per query (amino acids, or nucleotides on
// the forward strand) and a database searched on one strand.
static bool shard_query_codes( p_query * queries, size_t n, std::vector<QueryCodes> & qc, const char * who ) {
    const Config & c = config();
    if( c.symtype != AMINOACID && !(c.symtype == NUCLEOTIDE && c.strands == FORWARD_STRAND) ) {
        print_error( "%s: database-sharded searches take amino-acid or forward-strand nucleotide queries", who );
        return false;
    }
    for( size_t i = 0; i < n; i++ ) {
        test_configuration( queries[i] );
        if( queries[i]->symtype != c.symtype )
            fatal( "Query was read with a different symbol type than the current one." );
        if( queries[i]->len == 0 )
            fatal( "Query sequence is empty." );
        const QueryFrame & f = (*queries[i]->frames)[0];
        qc.push_back( QueryCodes{ (const uint8_t *) f.seq.data(), (uint32_t) (f.seq.size() - 1) } );
    }
    return true;
}

int ssa_b200_shard_scores( int algorithm, p_query * queries, size_t n_queries, int bit_width, size_t id_lo,
        size_t id_hi, int64_t * scores, int32_t * blocks_entry, int32_t * blocks_16 ) {
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH ) {
        print_error( "ssa_b200_shard_scores: unknown algorithm %d", algorithm );
        return -1;
    }
    if( id_lo > id_hi || id_hi > UINT32_MAX ) {
        print_error( "ssa_b200_shard_scores: bad record range [%zu, %zu)", id_lo, id_hi );
        return -1;
    }
    if( n_queries && id_hi > id_lo && (!queries || !scores || !blocks_entry || !blocks_16) ) {
        print_error( "ssa_b200_shard_scores: null array" );
        return -1;
    }
    std::vector<QueryCodes> qc;
    if( !shard_query_codes( queries, n_queries, qc, "ssa_b200_shard_scores" ) )
        return -1;
    SearchRequest req = make_request( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, 1, bit_width, COMPUTE_SCORE );
    SearchStats st;
    engine_shard_scores( req, qc, (uint32_t) id_lo, (uint32_t) id_hi, scores, blocks_entry, blocks_16, st );
    g_last_stats = st;
    return 0;
}

int ssa_b200_replay_gathered( int algorithm, p_query * queries, size_t n_queries, size_t hitcount, int bit_width,
        int align_type, const int64_t * scores, const int32_t * blocks_entry, const int32_t * blocks_16,
        p_alignment_list * results ) {
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH ) {
        print_error( "ssa_b200_replay_gathered: unknown algorithm %d", algorithm );
        return -1;
    }
    if( n_queries && (!queries || !results) ) {
        print_error( "ssa_b200_replay_gathered: null array" );
        return -1;
    }
    std::vector<QueryCodes> qc;
    if( !shard_query_codes( queries, n_queries, qc, "ssa_b200_replay_gathered" ) )
        return -1;
    SearchRequest req = make_request( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, hitcount, bit_width, align_type );
    HostDb db;
    lengths_db( db );
    const size_t n = db.n_ids;
    if( n && n_queries && (!scores || !blocks_entry || !blocks_16) ) {
        print_error( "ssa_b200_replay_gathered: null array" );
        return -1;
    }
    std::vector<uint32_t> rank;
    if( bit_width != BIT_WIDTH_64 )
        schedule_ranks( db, req.chunk_size, bit_width == BIT_WIDTH_8 ? req.lanes8 : req.lanes16, rank );
    std::vector<std::vector<Hit>> hits( n_queries );
    SearchStats st;
    st.query_overflow.assign( n_queries, { 0, 0 } );
    std::vector<int32_t> s32( n );
    for( size_t q = 0; q < n_queries; q++ ) {
        const int64_t * row = scores + q * n;
        ReplayQuery rq;
        for( size_t id = 0; id < n; id++ ) {
            const int64_t v = row[id];
            s32[id] = (v > INT32_MIN && v <= INT32_MAX) ? (int32_t) v : REPLAY_SCORE_IN_WIDE;
            if( blocks_entry[q * n + id] >= 0 )
                rq.ovf_entry.emplace_back( (uint32_t) id, blocks_entry[q * n + id] );
            if( blocks_16[q * n + id] >= 0 )
                rq.ovf16.emplace_back( (uint32_t) id, blocks_16[q * n + id] );
        }
        rq.score = s32.data();
        rq.score64 = row;
        ReplayCounts counts;
        replay_query( db, req, rq, rank.empty() ? nullptr : rank.data(), hits[q], counts );
        st.overflow8 += counts.overflow8;
        st.overflow16 += counts.overflow16;
        st.query_overflow[q] = { counts.overflow8, counts.overflow16 };
    }
    if( align_type == COMPUTE_ALIGNMENT )
        engine_align_hits( req, qc, hits, st );
    g_last_stats = st;
    for( size_t i = 0; i < n_queries; i++ )
        results[i] = make_list( hits[i], queries[i], align_type == COMPUTE_ALIGNMENT );
    return 0;
}

size_t ssa_b200_tuning_report( char * buf, size_t n ) {
    const std::string r = tuning_report();
    if( buf && n ) {
        const size_t m = std::min( n - 1, r.size() );
        memcpy( buf, r.data(), m );
        buf[m] = 0;
    }
    return r.size() + 1;
}

size_t ssa_b200_query_overflows( uint64_t * overflow_8_to_16, uint64_t * overflow_16_to_64, size_t n ) {
    const auto & q = g_last_stats.query_overflow;
    const size_t m = std::min( n, q.size() );
    for( size_t i = 0; i < m; i++ ) {
        if( overflow_8_to_16 )
            overflow_8_to_16[i] = q[i].first;
        if( overflow_16_to_64 )
            overflow_16_to_64[i] = q[i].second;
    }
    return q.size();
}

void ssa_db_refresh( void ) {
    engine_invalidate_database();
}

size_t ssa_query_length( p_query p ) {
    return p ? p->len : 0;
}

int ssa_b200_translation_table( int code, uint8_t * out ) {
    if( code < 1 || code > 25 || !NCBI_CODES[code - 1] || !out )
        return -1;
    translation_table( code, out );
    return 0;
}

struct ssa_server {
    ServerImpl impl;
};

ssa_server * ssa_server_start( int algorithm, size_t hitcount, int bit_width, int align_type, size_t slots,
        size_t segments, size_t memory_budget ) {
    if( algorithm != SSA_SMITH_WATERMAN && algorithm != SSA_NEEDLEMAN_WUNSCH )
        fatal( "\nUnknown search type: %d\n\n", algorithm );
    if( slots == 0 || slots > 4096 )
        fatal( "Server slots must be in 1..4096 (got %zu).", slots );
    const Config & c = config();
    if( !c.matrix_set )
        fatal( "Scoring not initialized." );
    if( !c.constant_scoring && c.symtype == NUCLEOTIDE )
        fatal( "Nucleotide sequences can only be aligned using constant scores." );
    if( !(c.symtype == AMINOACID || (c.symtype == NUCLEOTIDE && c.strands == FORWARD_STRAND)) )
        fatal( "The server runs protein and forward-strand nucleotide searches only." );
    if( engine_streaming() )
        fatal( "The server keeps the database resident in device memory; this database is larger than the "
                "database memory budget (ssa_b200_set_db_memory)." );
    ssa_server * sv = new ssa_server();
    ServerImpl & s = sv->impl;
    s.req = make_request( algorithm == SSA_SMITH_WATERMAN ? 0 : 1, hitcount, bit_width, align_type );
    s.matrix.assign( c.matrix, c.matrix + 1024 );
    s.req.matrix = s.matrix.data();
    s.slots = (uint32_t) slots;
    s.budget = memory_budget;
    s.owner.assign( slots, nullptr );
    s.seg = engine_serve_open( s.req, (uint32_t) slots, (uint32_t) std::max<size_t>( 1, segments ) );
    {
        const HostDb & db = engine_database();
        for( uint32_t l : db.len )
            s.max_db_len = std::max<uint64_t>( s.max_db_len, l );
        s.residues = db.residues;
    }
    s.loop_thread = std::thread( [&s] { s.loop(); } );
    return sv;
}

long long ssa_server_submit( ssa_server * sv, p_query query ) {
    if( !sv || !query )
        fatal( "Query not initialized." );
    ServerImpl & s = sv->impl;
    if( query->symtype != config().symtype )
        fatal( "Query was read with a different symbol type than the current one." );
    if( query->len == 0 || query->len > SERVE_MAX_QUERY ) {
        print_error( "Served queries must have 1..%u residues (got %zu).", SERVE_MAX_QUERY, query->len );
        return -1;
    }
    ServeTicket * t = new ServeTicket();
    t->query = query;
    // traceback memory of the request's hits, bounded by the longest sequence:
    // 2-bit directions (16 bits per 8 query rows and column), last rows, ops
    if( s.req.align_type == COMPUTE_ALIGNMENT )
        t->mem = (uint64_t) s.req.hitcount * (((query->len + 7) / 8) * 2 * s.max_db_len + 8 * query->len +
                query->len + s.max_db_len);
    t->t_submit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk( s.m );
        if( s.stopping ) {
            delete t;
            return -1;
        }
        t->id = s.next_id++;
        s.tickets[t->id] = t;
        s.pending.push_back( t );
        s.submitted++;
    }
    s.cv_work.notify_one();
    return t->id;
}

p_alignment_list ssa_server_wait( ssa_server * sv, long long ticket, double * latency_seconds ) {
    if( !sv )
        return nullptr;
    ServerImpl & s = sv->impl;
    std::unique_lock<std::mutex> lk( s.m );
    auto it = s.tickets.find( ticket );
    if( it == s.tickets.end() )
        return nullptr;
    ServeTicket * t = it->second;
    s.cv_done.wait( lk, [&] { return t->done; } );
    p_alignment_list r = t->result;
    if( latency_seconds )
        *latency_seconds = std::chrono::duration<double>( t->t_done - t->t_submit ).count();
    s.tickets.erase( it );
    delete t;
    return r;
}

void ssa_server_get_stats( ssa_server * sv, ssa_server_stats_t * out ) {
    if( !sv || !out )
        return;
    ServerImpl & s = sv->impl;
    std::lock_guard<std::mutex> lk( s.m );
    out->submitted = s.submitted;
    out->completed = s.completed;
    out->waves = s.waves;
    out->cells = s.cells;
    out->busy_seconds = s.busy_seconds;
    out->device_seconds = s.device_seconds;
    out->slots = s.slots;
    out->segments = (uint32_t) s.seg.size() - 1;
    out->queued = s.queued;
    out->slot_waves = s.slot_waves;
    out->max_pending = s.max_pending;
    out->max_occupied = s.max_occupied;
}

void ssa_server_stop( ssa_server * sv ) {
    if( !sv )
        return;
    ServerImpl & s = sv->impl;
    {
        std::lock_guard<std::mutex> lk( s.m );
        s.stopping = true;
    }
    s.cv_work.notify_all();
    if( s.loop_thread.joinable() )
        s.loop_thread.join();
    for( auto & kv : s.tickets ) {      // results nobody waited for
        if( kv.second->result )
            free_alignment( kv.second->result );
        delete kv.second;
    }
    delete sv;
}

}  // extern "C"
#pragma GCC visibility pop
