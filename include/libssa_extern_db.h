/*
 * libssa_extern_db.h -- the database plugin interface imported by libssa.
 *
 * libssa does not read sequence files itself.  It asks a database library for
 * sequences through these four functions, exactly as the CPU libssa does
 * (reference: src/libssa_extern_db.h:28-56).  The B200 build calls them once
 * per init_db() to pack the whole database into HBM, and again for each hit it
 * materialises (reference: src/algo/aligner.c:65).
 *
 * Contract (unchanged from the reference):
 *   - IDs are 0-based and dense: ssa_db_get_sequence(i) for i < count returns a
 *     record whose ID is i; it returns NULL for i >= count.
 *   - seq holds raw ASCII residues (upper or lower case), seqlen bytes long.
 *   - Returned records are owned by the database library and stay valid until
 *     ssa_db_close().
 */
#ifndef LIBSSA_EXTERN_DB_H_
#define LIBSSA_EXTERN_DB_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    size_t ID;
    size_t seqlen;
    char * seq;
} seqinfo_t;

typedef seqinfo_t * p_seqinfo;

/* Opens the database named by db_name (reference: src/libssa_extern_db.h:39). */
int ssa_db_init( const char * db_name );

/* Number of records, including empty ones (reference: src/libssa_extern_db.h:44). */
size_t ssa_db_get_sequence_count( void );

/* Record with the given 0-based ID, or NULL past the end
 * (reference: src/libssa_extern_db.h:49). */
p_seqinfo ssa_db_get_sequence( size_t id );

/* Releases everything ssa_db_init allocated (reference: src/libssa_extern_db.h:56). */
void ssa_db_close( void );

#ifdef __cplusplus
}
#endif

#endif /* LIBSSA_EXTERN_DB_H_ */
