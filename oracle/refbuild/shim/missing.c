/*
 * missing.c -- a function the reference's sources call without defining it
 * in a build without hwloc: common/isched_nohwloc.c names pastix_warning,
 * which no file of the reference provides.  It prints the message to stderr.
 * TEST INFRASTRUCTURE ONLY (oracle build).
 */
#include <stdarg.h>
#include <stdio.h>

void pastix_warning( const char *fmt, ... )
{
    va_list ap;
    va_start( ap, fmt );
    fprintf( stderr, "pastix warning: " );
    vfprintf( stderr, fmt, ap );
    fprintf( stderr, "\n" );
    va_end( ap );
}
