/*
 * A client of the libssa C API, written the way the reference's own callers
 * are (src/libssa_example.c, tests/test_libssa.c:30-93): configure, load a
 * database, read a query, search, walk the returned list, free.  It compiles
 * unchanged against the reference's libssa.h and links against either
 * library.
 *
 *     search_example <db.fasta> <query.fasta>
 *
 * Prints one line per hit: algorithm, ID, score, CIGAR and coordinates.
 */
#include <stdio.h>

#include "libssa.h"

static void print_list( const char * algo, p_alignment_list list ) {
    for( size_t i = 0; i < list->len; i++ ) {
        alignment_t * a = list->alignments[i];
        printf( "%s %zu %ld %s %zu %zu %zu %zu\n", algo, a->db_seq.ID, a->score,
                a->alignment ? a->alignment : "-", a->align_q_start, a->align_q_end, a->align_d_start,
                a->align_d_end );
    }
}

int main( int argc, char ** argv ) {
    if( argc != 3 ) {
        fprintf( stderr, "usage: %s <db.fasta> <query.fasta>\n", argv[0] );
        return 2;
    }
    set_output_mode( OUTPUT_SILENT );
    set_thread_count( 1 );
    set_simd_compute_mode( COMPUTE_ON_AVX2 );
    init_symbol_translation( NUCLEOTIDE, FORWARD_STRAND, 3, 3 );
    init_constant_scores( 5, -4 );
    init_gap_penalties( -4, -2 );
    init_db( argv[1] );

    p_query query = init_sequence_fasta( READ_FROM_FILE, argv[2] );
    if( !query )
        return 1;

    p_alignment_list sw = sw_align( query, 5, BIT_WIDTH_64, COMPUTE_ALIGNMENT );
    print_list( "sw", sw );
    free_alignment( sw );

    p_alignment_list nw = nw_align( query, 5, BIT_WIDTH_64, COMPUTE_ALIGNMENT );
    print_list( "nw", nw );
    free_alignment( nw );

    free_sequence( query );
    ssa_exit();
    return 0;
}
