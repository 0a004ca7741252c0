/*
 * ref_run.c -- command-line driver around the reference libssa, built from
 * the reference's own sources by oracle/Makefile into oracle/_ref/ref_run.
 *
 * TEST INFRASTRUCTURE ONLY.  This program is the oracle's ground truth: it
 * runs the unmodified CPU libssa through its public API (reference:
 * src/libssa.h:122-263) and prints what it returns.  Tests, the golden-fixture
 * generator and bench.py's CPU-baseline leg execute it; the product never
 * does.
 *
 * Usage:
 *   ref_run [options] --db DB --queries FASTA --out OUT.json
 *   ref_run --dump-matrix SPEC            (prints the 32x32 int64 table)
 *   ref_run --dump-translation CODE       (prints the amino-acid code of every
 *                                          nucleotide triple (a,b,c), codes 0-15,
 *                                          under genetic code CODE, 4096 values)
 *
 * Options:
 *   --algo sw|nw        --width 8|16|64     --align 0|1     --hits K
 *   --symtype T         --strands S         --gencode Q,D
 *   --matrix builtin:NAME | const:MATCH,MISMATCH | file:PATH
 *   --gap O,E           --chunk C           --threads T     --simd M
 *   --max-queries N     --repeat R          --time
 *
 * For every query record of the FASTA file ref_run calls
 * init_sequence_fasta(READ_FROM_STRING, seq), sw_align/nw_align and writes one
 * JSON object per line to OUT.json with the hits (score, ID, CIGAR,
 * coordinates), the 8->16 and 16->64 overflow counts the library reports, and
 * the wall time of the align call.  With --time messages are silenced and
 * only timings are meaningful.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>

#include "libssa.h"
#include "matrices.h"
#include "util/util_sequence.h"

static double now_s( void ) {
    struct timespec ts;
    clock_gettime( CLOCK_MONOTONIC, &ts );
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void apply_matrix( const char * spec ) {
    if( strncmp( spec, "builtin:", 8 ) == 0 ) {
        init_score_matrix( MATRIX_BUILDIN, spec + 8 );
    }
    else if( strncmp( spec, "const:", 6 ) == 0 ) {
        int match = 0, mismatch = 0;
        if( sscanf( spec + 6, "%d,%d", &match, &mismatch ) != 2 ) {
            fprintf( stderr, "bad --matrix %s\n", spec );
            exit( 2 );
        }
        init_constant_scores( (int8_t) match, (int8_t) mismatch );
    }
    else if( strncmp( spec, "file:", 5 ) == 0 ) {
        init_score_matrix( READ_FROM_FILE, spec + 5 );
    }
    else {
        fprintf( stderr, "bad --matrix %s\n", spec );
        exit( 2 );
    }
}

/* Reads all records of a FASTA file: returns the count, fills *seqs. */
static size_t read_queries( const char * path, char *** seqs_out ) {
    FILE * fp = fopen( path, "rb" );
    if( !fp ) {
        fprintf( stderr, "cannot open %s\n", path );
        exit( 2 );
    }
    size_t cap = 16, n = 0;
    char ** seqs = malloc( cap * sizeof(char*) );
    char * cur = NULL;
    size_t clen = 0, ccap = 0;
    char * line = NULL;
    size_t lcap = 0;
    ssize_t got;
    while( (got = getline( &line, &lcap, fp )) >= 0 ) {
        if( got > 0 && line[0] == '>' ) {
            if( cur ) {
                if( n == cap ) {
                    cap *= 2;
                    seqs = realloc( seqs, cap * sizeof(char*) );
                }
                seqs[n++] = cur;
            }
            ccap = 256;
            clen = 0;
            cur = malloc( ccap );
            cur[0] = 0;
            continue;
        }
        if( !cur )
            continue;
        for( ssize_t i = 0; i < got; i++ ) {
            char c = line[i];
            if( c == '\n' || c == '\r' )
                continue;
            if( clen + 2 >= ccap ) {
                ccap *= 2;
                cur = realloc( cur, ccap );
            }
            cur[clen++] = c;
            cur[clen] = 0;
        }
    }
    if( cur ) {
        if( n == cap ) {
            cap *= 2;
            seqs = realloc( seqs, cap * sizeof(char*) );
        }
        seqs[n++] = cur;
    }
    free( line );
    fclose( fp );
    *seqs_out = seqs;
    return n;
}

static void json_string( FILE * out, const char * s ) {
    fputc( '"', out );
    for( ; s && *s; s++ ) {
        if( *s == '"' || *s == '\\' )
            fputc( '\\', out );
        fputc( *s, out );
    }
    fputc( '"', out );
}

/* Runs fn with stdout redirected to a temporary file and scans the
 * library's "Overflow occurred: A ... B" info line. */
static p_alignment_list run_captured( p_alignment_list (*fn)( p_query, size_t, int, int ), p_query q, size_t hits,
        int width, int align, long * ovf8, long * ovf16 ) {
    char tmpl[] = "/tmp/ref_run_XXXXXX";
    int fd = mkstemp( tmpl );
    fflush( stdout );
    int saved = dup( 1 );
    dup2( fd, 1 );
    p_alignment_list l = fn( q, hits, width, align );
    fflush( stdout );
    dup2( saved, 1 );
    close( saved );
    lseek( fd, 0, SEEK_SET );
    FILE * f = fdopen( fd, "r" );
    char buf[4096];
    *ovf8 = 0;
    *ovf16 = 0;
    while( fgets( buf, sizeof(buf), f ) ) {
        char * p = strstr( buf, "Overflow occurred: " );
        if( p ) {
            sscanf( p, "Overflow occurred: %ld sequences were re-aligned with 16 bit, and %ld", ovf8, ovf16 );
        }
    }
    fclose( f );
    unlink( tmpl );
    return l;
}

int main( int argc, char ** argv ) {
    const char * algo = "sw";
    int width = 8, align = 1, symtype = AMINOACID, strands = FORWARD_STRAND;
    int qgc = 1, dgc = 1, simd = COMPUTE_ON_AVX2, timing = 0;
    long hits = 10, chunk = 1000, threads = 1, max_queries = -1, repeat = 1;
    int gap_o = -11, gap_e = -1;
    const char * matrix = "builtin:blosum62";
    const char * db = NULL, * queries = NULL, * out_path = NULL;

    for( int i = 1; i < argc; i++ ) {
        const char * a = argv[i];
        const char * v = (i + 1 < argc) ? argv[i + 1] : "";
        if( !strcmp( a, "--dump-matrix" ) ) {
            apply_matrix( v );
            printf( "[" );
            for( int k = 0; k < SCORE_MATRIX_DIM * SCORE_MATRIX_DIM; k++ )
                printf( "%s%ld", k ? "," : "", (long) score_matrix_64[k] );
            printf( "]\n" );
            return 0;
        }
        else if( !strcmp( a, "--dump-translation" ) ) {
            // translate the 4096 nucleotide triples with the reference's own
            // translation of a query sequence (frame 0, forward strand)
            const int gc = atoi( v );
            us_init_translation( gc, gc );
            sequence_t dna = { malloc( 3 * 4096 + 1 ), 3 * 4096 };
            for( int t = 0; t < 4096; t++ ) {
                dna.seq[3 * t] = (char) (t >> 8);
                dna.seq[3 * t + 1] = (char) ((t >> 4) & 15);
                dna.seq[3 * t + 2] = (char) (t & 15);
            }
            sequence_t prot = { NULL, 0 };
            us_translate_sequence( 0, dna, 0, 0, &prot );
            printf( "[" );
            for( size_t k = 0; k < prot.len; k++ )
                printf( "%s%d", k ? "," : "", (int) prot.seq[k] );
            printf( "]\n" );
            return 0;
        }
        else if( !strcmp( a, "--algo" ) ) { algo = v; i++; }
        else if( !strcmp( a, "--width" ) ) { width = atoi( v ); i++; }
        else if( !strcmp( a, "--align" ) ) { align = atoi( v ); i++; }
        else if( !strcmp( a, "--hits" ) ) { hits = atol( v ); i++; }
        else if( !strcmp( a, "--symtype" ) ) { symtype = atoi( v ); i++; }
        else if( !strcmp( a, "--strands" ) ) { strands = atoi( v ); i++; }
        else if( !strcmp( a, "--gencode" ) ) { sscanf( v, "%d,%d", &qgc, &dgc ); i++; }
        else if( !strcmp( a, "--matrix" ) ) { matrix = v; i++; }
        else if( !strcmp( a, "--gap" ) ) { sscanf( v, "%d,%d", &gap_o, &gap_e ); i++; }
        else if( !strcmp( a, "--chunk" ) ) { chunk = atol( v ); i++; }
        else if( !strcmp( a, "--threads" ) ) { threads = atol( v ); i++; }
        else if( !strcmp( a, "--simd" ) ) { simd = atoi( v ); i++; }
        else if( !strcmp( a, "--db" ) ) { db = v; i++; }
        else if( !strcmp( a, "--queries" ) ) { queries = v; i++; }
        else if( !strcmp( a, "--out" ) ) { out_path = v; i++; }
        else if( !strcmp( a, "--max-queries" ) ) { max_queries = atol( v ); i++; }
        else if( !strcmp( a, "--repeat" ) ) { repeat = atol( v ); i++; }
        else if( !strcmp( a, "--time" ) ) { timing = 1; }
        else {
            fprintf( stderr, "unknown option %s\n", a );
            return 2;
        }
    }
    if( !db || !queries || !out_path ) {
        fprintf( stderr, "need --db, --queries and --out\n" );
        return 2;
    }

    set_output_mode( timing ? OUTPUT_SILENT : OUTPUT_INFO );
    set_simd_compute_mode( simd );
    set_chunk_size( (size_t) chunk );
    set_thread_count( (size_t) threads );
    apply_matrix( matrix );
    init_gap_penalties( (int8_t) gap_o, (int8_t) gap_e );
    init_symbol_translation( symtype, strands, dgc, qgc );
    init_db( db );

    char ** seqs = NULL;
    size_t nq = read_queries( queries, &seqs );
    if( max_queries >= 0 && (size_t) max_queries < nq )
        nq = (size_t) max_queries;

    FILE * out = fopen( out_path, "w" );
    if( !out ) {
        fprintf( stderr, "cannot write %s\n", out_path );
        return 2;
    }
    p_alignment_list (*fn)( p_query, size_t, int, int ) = strcmp( algo, "nw" ) ? &sw_align : &nw_align;

    for( size_t qi = 0; qi < nq; qi++ ) {
        p_query q = init_sequence_fasta( READ_FROM_STRING, seqs[qi] );
        for( long r = 0; r < repeat; r++ ) {
            long ovf8 = -1, ovf16 = -1;
            double t0 = now_s();
            p_alignment_list l;
            if( timing )
                l = fn( q, (size_t) hits, width, align );
            else
                l = run_captured( fn, q, (size_t) hits, width, align, &ovf8, &ovf16 );
            double t1 = now_s();
            if( r == repeat - 1 ) {
                fprintf( out, "{\"qidx\":%zu,\"seconds\":%.9f,\"ovf8\":%ld,\"ovf16\":%ld,\"hits\":[", qi, t1 - t0, ovf8,
                        ovf16 );
                for( size_t h = 0; h < l->len; h++ ) {
                    p_alignment a = l->alignments[h];
                    fprintf( out, "%s{\"id\":%zu,\"score\":%ld,\"dlen\":%zu,\"qlen\":%zu,\"q_start\":%zu,\"q_end\":%zu,"
                            "\"d_start\":%zu,\"d_end\":%zu,\"strand\":%d,\"frame\":%d,\"qstrand\":%d,\"qframe\":%d,"
                            "\"alignment_len\":%zu,\"cigar\":",
                            h ? "," : "", a->db_seq.ID, a->score, a->db_seq.len, a->query.len, a->align_q_start,
                            a->align_q_end, a->align_d_start, a->align_d_end, a->db_seq.strand, a->db_seq.frame,
                            a->query.strand, a->query.frame, a->alignment ? a->alignment_len : 0 );
                    if( a->alignment )
                        json_string( out, a->alignment );
                    else
                        fputs( "null", out );
                    fputc( '}', out );
                }
                fputs( "]}\n", out );
            }
            else {
                fprintf( out, "{\"qidx\":%zu,\"seconds\":%.9f,\"warmup\":true}\n", qi, t1 - t0 );
            }
            free_alignment( l );
        }
        free_sequence( q );
        fflush( out );
    }
    fclose( out );
    ssa_exit();
    return 0;
}
