/* wave_stats.c -- the reference daligner with its own wave counters switched on.
 *
 * Test and measurement infrastructure only; nothing of it ships.  oracle/Makefile writes
 * oracle/_ref/align_wavestats.c, the reference's dalign/align.c with its "#undef
 * WAVE_STATS" line (dalign/align.c:44) turned into "#define WAVE_STATS", and links this
 * file -- which includes that copy, so that the counters' file statics are in scope --
 * with the reference's dalign/daligner.c and dalign/filter.c into
 * oracle/_ref/daligner_wavestats.  With WAVE_STATS every forward and reverse wave adds its
 * width hgh - low + 1 to TOT and 1 to NWV (dalign/align.c:957-963, 1694-1700): TOT is the
 * aligner's cell count, the unit of GCUPS.  The reference never prints them from
 * daligner, so an exit handler writes them to stderr:
 *
 *     WAVE_STATS cells <TOT> waves <NWV> widest <MAX>
 *
 * The counters are plain int64 additions shared by all threads: exact with -j1 only.
 */
#include "align_wavestats.c"

static void wave_stats_report(void)
{
    fprintf(stderr, "WAVE_STATS cells %lld waves %lld widest %lld\n", (long long)TOT, (long long)NWV, (long long)MAX);
}

__attribute__((constructor)) static void wave_stats_register(void)
{
    atexit(wave_stats_report);
}
