// tuning.cpp -- the measured shape table the entry passes choose their tile
// shapes from.
//
// The reference fixes its tile: 4-column blocks (CDEPTH) and 32 or 16 lanes
// per vector (src/algo/8/search_8_util.h:25-27, src/algo/8/search_8.c:41-56).
// The B200 entry kernels have free shape parameters instead -- rows per
// thread R and resident CTAs per SM of the query-pair kernel, threads per
// sequence G, rows per thread R and columns per step of the single-query
// kernel -- whose best values depend on the query length (padding to whole
// passes) and on the database (wavefront fill per sequence, occupancy).
// libssa_b200/tune.py times every candidate on the device and writes the
// measured cost of a unit of work per candidate and database bucket into a
// text file; the engine reads it once and picks, per query, the shape with
// the smallest passes x cost.
//
// File format (one entry per line, '#' starts a comment):
//   version <n>
//   device <name ...>
//   qpair <bucket> <R> <MB> <ps per query pair, pass and database column>
//   qpair4 <bucket> <R> <MB> <ps ...>       (the kernel with 4 columns per step)
//   qpair4h <bucket> <R> <MB> <ps ...>      (4 columns, running maximum in fp16x2)
//   qpair4g8 <bucket> 24 <MB> <ps ...>      (4 columns, 96-row passes as 8 threads of 12 rows)
//   fast <bucket> <G> <R> <ps per pass and database column>
//   fast4 <bucket> <G> <R> <ps ...>          (the single-query kernel with 4 columns per step)
// Buckets: db_bucket() below.  Missing entries fall back to the built-in
// costs (measured the same way on a B200 before the tuner existed).
#include "ssa_internal.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <string>

namespace ssa {

namespace {

TuningTable g_table;
std::once_flag g_once;

// The built-in relative costs of the query-pair kernel per pass (64 queries of
// 375 residues against 10,000 sequences, each R pinned, 4 CTAs per SM).
void builtin( TuningTable & t ) {
    static const double cost[4] = { 4.28, 3.77, 4.56, 5.41 };
    for( int b = 0; b < TUNE_BUCKETS; b++ )
        for( int ri = 0; ri < 4; ri++ )
            t.qpair[b][ri][0][0] = cost[ri];
}

std::string default_path() {
    // <package>/tuning/b200.tune beside <package>/_lib/libssa.so
    Dl_info info;
    if( dladdr( (void *) &default_path, &info ) && info.dli_fname ) {
        std::string so = info.dli_fname;
        const size_t slash = so.rfind( '/' );
        if( slash != std::string::npos ) {
            std::string dir = so.substr( 0, slash );
            const size_t up = dir.rfind( '/' );
            if( up != std::string::npos )
                return dir.substr( 0, up ) + "/tuning/b200.tune";
        }
    }
    return "";
}

void load( TuningTable & t ) {
    builtin( t );
    const char * env = getenv( "SSA_B200_TUNING" );
    if( env && strcmp( env, "builtin" ) == 0 )
        return;
    const std::string path = env ? std::string( env ) : default_path();
    FILE * f = path.empty() ? nullptr : fopen( path.c_str(), "r" );
    if( !f )
        return;
    char line[512];
    bool any = false;
    while( fgets( line, sizeof line, f ) ) {
        char * hash = strchr( line, '#' );
        if( hash )
            *hash = 0;
        char key[32] = { 0 };
        if( sscanf( line, "%31s", key ) != 1 )
            continue;
        if( !strcmp( key, "version" ) ) {
            sscanf( line, "%*s %d", &t.version );
        }
        else if( !strcmp( key, "device" ) ) {
            const char * p = line + strlen( "device" );
            while( *p == ' ' || *p == '\t' )
                p++;
            t.device = p;
            while( !t.device.empty() && (t.device.back() == '\n' || t.device.back() == '\r' || t.device.back() == ' ') )
                t.device.pop_back();
        }
        else if( !strcmp( key, "qpair" ) || !strcmp( key, "qpair4" ) || !strcmp( key, "qpair4h" ) ||
                !strcmp( key, "qpair4g8" ) ) {
            const int ci = !strcmp( key, "qpair" ) ? 0 : !strcmp( key, "qpair4" ) ? 1 : !strcmp( key, "qpair4h" ) ? 2 : 3;
            if( ci == 3 && strstr( line, " 24 " ) == nullptr )
                continue;
            int b, R, mb;
            double ps;
            if( sscanf( line, "%*s %d %d %d %lf", &b, &R, &mb, &ps ) == 4 && b >= 0 && b < TUNE_BUCKETS &&
                    R >= 16 && R <= 28 && R % 4 == 0 && (mb == 4 || mb == 5) && ps > 0 ) {
                if( !any ) {
                    // a measured table replaces the built-in costs entirely
                    memset( t.qpair, 0, sizeof t.qpair );
                    any = true;
                }
                t.qpair[b][R / 4 - 4][mb - 4][ci] = ps;
            }
        }
        else if( !strcmp( key, "fast" ) ) {
            int b, G, R;
            double ps;
            if( sscanf( line, "%*s %d %d %d %lf", &b, &G, &R, &ps ) == 4 && b >= 0 && b < TUNE_BUCKETS &&
                    (G == 8 || G == 16 || G == 32) && R >= 8 && R <= 32 && R % 8 == 0 && ps > 0 ) {
                const int gi = G == 8 ? 0 : G == 16 ? 1 : 2;
                t.fast[b][gi][R / 8 - 1] = ps;
                t.has_fast = true;
            }
        }
        else if( !strcmp( key, "fast4" ) ) {
            int b, G, R;
            double ps;
            if( sscanf( line, "%*s %d %d %d %lf", &b, &G, &R, &ps ) == 4 && b >= 0 && b < TUNE_BUCKETS &&
                    (G == 4 || G == 8 || G == 16 || G == 32) && R >= 8 && R <= 24 && R % 8 == 0 && ps > 0 ) {
                const int gi = G == 4 ? 0 : G == 8 ? 1 : G == 16 ? 2 : 3;
                t.fast4[b][gi][R / 8 - 1] = ps;
                t.has_fast4 = true;
            }
        }
    }
    fclose( f );
    t.source = path;
}

}  // namespace

const TuningTable & tuning() {
    std::call_once( g_once, [] { load( g_table ); } );
    return g_table;
}

int db_bucket( double mean_len, uint64_t n_seqs ) {
    const int len_b = mean_len < 250.0 ? 0 : mean_len < 1000.0 ? 1 : 2;
    return len_b + (n_seqs < 50000 ? 0 : 3);
}

}  // namespace ssa
