/*
 * Prints, as JSON, the sizes and field offsets of the libssa.h and
 * libssa_extern_db.h types and the values of the libssa.h constants, as seen
 * by a C compiler through whichever header directory it is built with.  Built
 * against the reference's headers it produced tests/golden/abi_layout.json;
 * built against include/ it must print the same.
 */
#include <stddef.h>
#include <stdio.h>

#include "libssa.h"
#include "libssa_extern_db.h"

#define FIELD( T, m ) printf( "  \"%s.%s\": [%zu, %zu],\n", #T, #m, offsetof( T, m ), sizeof( ((T *) 0)->m ) )
#define SIZE( T ) printf( "  \"sizeof(%s)\": %zu,\n", #T, sizeof( T ) )
#define CONST( c ) printf( "  \"%s\": %d,\n", #c, (int) (c) )

int main( void ) {
    printf( "{\n" );
    SIZE( db_seq_t );
    FIELD( db_seq_t, seq );
    FIELD( db_seq_t, len );
    FIELD( db_seq_t, ID );
    FIELD( db_seq_t, strand );
    FIELD( db_seq_t, frame );
    SIZE( q_seq_t );
    FIELD( q_seq_t, seq );
    FIELD( q_seq_t, len );
    FIELD( q_seq_t, strand );
    FIELD( q_seq_t, frame );
    SIZE( alignment_t );
    FIELD( alignment_t, db_seq );
    FIELD( alignment_t, query );
    FIELD( alignment_t, alignment );
    FIELD( alignment_t, alignment_len );
    FIELD( alignment_t, score );
    FIELD( alignment_t, align_q_start );
    FIELD( alignment_t, align_q_end );
    FIELD( alignment_t, align_d_start );
    FIELD( alignment_t, align_d_end );
    SIZE( alignment_list_t );
    FIELD( alignment_list_t, alignments );
    FIELD( alignment_list_t, len );
    SIZE( seqinfo_t );
    FIELD( seqinfo_t, ID );
    FIELD( seqinfo_t, seqlen );
    FIELD( seqinfo_t, seq );
    CONST( NUCLEOTIDE );
    CONST( AMINOACID );
    CONST( TRANS_QUERY );
    CONST( TRANS_DB );
    CONST( TRANS_BOTH );
    CONST( FORWARD_STRAND );
    CONST( COMPLEMENTARY_STRAND );
    CONST( BOTH_STRANDS );
    CONST( BIT_WIDTH_8 );
    CONST( BIT_WIDTH_16 );
    CONST( BIT_WIDTH_64 );
    CONST( OUTPUT_SILENT );
    CONST( OUTPUT_ERROR );
    CONST( OUTPUT_WARNING );
    CONST( OUTPUT_INFO );
    CONST( COMPUTE_SCORE );
    CONST( COMPUTE_ALIGNMENT );
    CONST( READ_FROM_FILE );
    CONST( READ_FROM_STRING );
    CONST( MATRIX_BUILDIN );
    CONST( COMPUTE_ON_SSE2 );
    CONST( COMPUTE_ON_SSE41 );
    CONST( COMPUTE_ON_AVX2 );
    printf( "  \"end\": 0\n}\n" );
    return 0;
}
