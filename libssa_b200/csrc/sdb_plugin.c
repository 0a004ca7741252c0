/*
 * sdb_plugin.c -- a database library implementing libssa_extern_db.h.
 *
 * The CPU libssa links an external, separately distributed FASTA reader
 * ("libsdb") behind src/libssa_extern_db.h.  That library is not part of the
 * reference tree, so this file provides a self-contained implementation with
 * the same observable contract (reference: tests/test_libssa_extern_db.c:24-58):
 *
 *   - ssa_db_init(name) opens a FASTA file (records start with '>', the header
 *     line is ignored, sequence lines are concatenated without their line
 *     breaks) or, when the name ends in ".sdb", the binary layout below;
 *   - IDs are the 0-based record index in file order; empty records keep their
 *     ID and report seqlen 0;
 *   - ssa_db_get_sequence(id) returns NULL for id >= count.
 *
 * Binary ".sdb" layout (little endian): 8-byte magic "SSADB001", uint64 count,
 * uint64 lengths[count], then the residues of all records back to back.
 *
 * ssa_db_b200_load_memory() installs a database straight from memory, which is
 * how tests and benchmarks feed seeded synthetic databases without files.
 *
 * All storage is one contiguous NUL-separated residue buffer plus one
 * seqinfo_t per record, so every returned seq is also a C string.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "libssa_extern_db.h"

#if defined(__GNUC__)
#define SDB_EXPORT __attribute__((visibility("default")))
#else
#define SDB_EXPORT
#endif

static char * sdb_buffer = NULL;      /* residues, each record NUL-terminated */
static seqinfo_t * sdb_records = NULL;
static size_t sdb_count = 0;

static void sdb_reset( void ) {
    free( sdb_buffer );
    free( sdb_records );
    sdb_buffer = NULL;
    sdb_records = NULL;
    sdb_count = 0;
}

/* Builds the record table from a residue buffer and per-record lengths.  The
 * buffer must hold sum(len)+count bytes with each record already followed by
 * a NUL byte. */
static int sdb_index( char * buffer, const uint64_t * lengths, size_t count ) {
    sdb_records = (seqinfo_t *) calloc( count ? count : 1, sizeof(seqinfo_t) );
    if( !sdb_records ) {
        free( buffer );
        return -1;
    }
    size_t off = 0;
    for( size_t i = 0; i < count; i++ ) {
        sdb_records[i].ID = i;
        sdb_records[i].seqlen = (size_t) lengths[i];
        sdb_records[i].seq = buffer + off;
        off += (size_t) lengths[i] + 1;
    }
    sdb_buffer = buffer;
    sdb_count = count;
    return 0;
}

static int ends_with( const char * s, const char * suffix ) {
    size_t n = strlen( s ), m = strlen( suffix );
    return n >= m && strcmp( s + n - m, suffix ) == 0;
}

static int sdb_read_binary( FILE * fp ) {
    char magic[8];
    uint64_t count = 0;
    if( fread( magic, 1, 8, fp ) != 8 || memcmp( magic, "SSADB001", 8 ) != 0 )
        return -1;
    if( fread( &count, sizeof(count), 1, fp ) != 1 )
        return -1;
    uint64_t * lengths = (uint64_t *) malloc( (count ? count : 1) * sizeof(uint64_t) );
    if( !lengths )
        return -1;
    if( count && fread( lengths, sizeof(uint64_t), count, fp ) != count ) {
        free( lengths );
        return -1;
    }
    size_t total = 0;
    for( uint64_t i = 0; i < count; i++ )
        total += (size_t) lengths[i] + 1;
    char * buffer = (char *) malloc( total ? total : 1 );
    if( !buffer ) {
        free( lengths );
        return -1;
    }
    size_t off = 0;
    for( uint64_t i = 0; i < count; i++ ) {
        if( lengths[i] && fread( buffer + off, 1, lengths[i], fp ) != lengths[i] ) {
            free( buffer );
            free( lengths );
            return -1;
        }
        off += lengths[i];
        buffer[off++] = 0;
    }
    int rc = sdb_index( buffer, lengths, (size_t) count );
    free( lengths );
    return rc;
}

static int sdb_read_fasta( FILE * fp ) {
    size_t cap = 1 << 16, used = 0;
    size_t lcap = 1024, nrec = 0;
    char * buffer = (char *) malloc( cap );
    uint64_t * lengths = (uint64_t *) malloc( lcap * sizeof(uint64_t) );
    if( !buffer || !lengths ) {
        free( buffer );
        free( lengths );
        return -1;
    }
    int c;
    int at_line_start = 1;
    int in_header = 0;
    int have_record = 0;
    size_t rec_start = 0;
    while( (c = fgetc( fp )) != EOF ) {
        if( at_line_start && c == '>' ) {
            if( have_record ) {
                lengths[nrec - 1] = used - rec_start;
                buffer[used++] = 0;
            }
            if( nrec == lcap ) {
                lcap *= 2;
                uint64_t * nl = (uint64_t *) realloc( lengths, lcap * sizeof(uint64_t) );
                if( !nl ) {
                    free( buffer );
                    free( lengths );
                    return -1;
                }
                lengths = nl;
            }
            nrec++;
            have_record = 1;
            in_header = 1;
            rec_start = used;
            at_line_start = 0;
            continue;
        }
        if( c == '\n' ) {
            in_header = 0;
            at_line_start = 1;
            continue;
        }
        at_line_start = 0;
        if( in_header || !have_record || c == '\r' )
            continue;
        if( used + 2 >= cap ) {
            cap *= 2;
            char * nb = (char *) realloc( buffer, cap );
            if( !nb ) {
                free( buffer );
                free( lengths );
                return -1;
            }
            buffer = nb;
        }
        buffer[used++] = (char) c;
    }
    if( have_record ) {
        if( used + 1 >= cap ) {
            char * nb = (char *) realloc( buffer, used + 2 );
            if( !nb ) {
                free( buffer );
                free( lengths );
                return -1;
            }
            buffer = nb;
        }
        lengths[nrec - 1] = used - rec_start;
        buffer[used++] = 0;
    }
    int rc = sdb_index( buffer, lengths, nrec );
    free( lengths );
    return rc;
}

SDB_EXPORT int ssa_db_init( const char * db_name ) {
    sdb_reset();
    if( !db_name )
        return -1;
    FILE * fp = fopen( db_name, "rb" );
    if( !fp ) {
        fprintf( stderr, "sdb: cannot open database file: %s\n", db_name );
        return -1;
    }
    int rc = ends_with( db_name, ".sdb" ) ? sdb_read_binary( fp ) : sdb_read_fasta( fp );
    fclose( fp );
    if( rc != 0 ) {
        fprintf( stderr, "sdb: cannot parse database file: %s\n", db_name );
        sdb_reset();
    }
    return rc;
}

SDB_EXPORT size_t ssa_db_get_sequence_count( void ) {
    return sdb_count;
}

SDB_EXPORT p_seqinfo ssa_db_get_sequence( size_t id ) {
    if( id >= sdb_count )
        return NULL;
    return &sdb_records[id];
}

SDB_EXPORT void ssa_db_close( void ) {
    sdb_reset();
}

/* Installs a database from memory: record i is residues[offsets[i] ..
 * offsets[i+1]).  The data is copied.  Returns 0 on success. */
SDB_EXPORT int ssa_db_b200_load_memory( size_t count, const char * residues, const uint64_t * offsets ) {
    sdb_reset();
    uint64_t * lengths = (uint64_t *) malloc( (count ? count : 1) * sizeof(uint64_t) );
    if( !lengths )
        return -1;
    size_t total = 0;
    for( size_t i = 0; i < count; i++ ) {
        lengths[i] = offsets[i + 1] - offsets[i];
        total += (size_t) lengths[i] + 1;
    }
    char * buffer = (char *) malloc( total ? total : 1 );
    if( !buffer ) {
        free( lengths );
        return -1;
    }
    size_t off = 0;
    for( size_t i = 0; i < count; i++ ) {
        memcpy( buffer + off, residues + offsets[i], (size_t) lengths[i] );
        off += (size_t) lengths[i];
        buffer[off++] = 0;
    }
    int rc = sdb_index( buffer, lengths, count );
    free( lengths );
    return rc;
}
