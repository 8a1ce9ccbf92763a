/* gd_report.c -- daligner's -v report and index-size warning (see gd_report.h). */
#include "gd_report.h"

#include <math.h>
#include <stdio.h>

void gd_report_number(int64_t num, int width)
{
    char t[48];
    long long n = (long long)num;
    if (n < 1000ll)
        snprintf(t, sizeof t, "%lld", n);
    else if (n < 1000000ll)
        snprintf(t, sizeof t, "%lld,%03lld", n / 1000ll, n % 1000ll);
    else if (n < 1000000000ll)
        snprintf(t, sizeof t, "%lld,%03lld,%03lld", n / 1000000ll, (n % 1000000ll) / 1000ll, n % 1000ll);
    else
        snprintf(t, sizeof t, "%lld,%03lld,%03lld,%03lld", n / 1000000000ll, (n % 1000000000ll) / 1000000ll,
                 (n % 1000000ll) / 1000ll, n % 1000ll);
    printf("%*s", width, t);
}

void gd_report_index(gd_context* ctx, int slot, int64_t slots, int suppress, int64_t mem_limit, int mem_physical,
                     int verbose)
{
    if (slots <= 0)
        return;
    gd_stats st;
    gd_get_stats(ctx, &st);
    const int64_t kmers = st.kmers[slot];
    if (verbose)
    {
        printf("\n   Kmer count = ");
        gd_report_number(slots, 0);
        printf("\n   Using %.2fGb of space\n", (1. * slots) / 33554432);
        if (suppress > 0)
        {
            printf("   Revised kmer count = ");
            gd_report_number(kmers, 0);
            printf("\n");
        }
        printf("   Index occupies %.2fGb\n", (1. * kmers) / 67108864);
        fflush(stdout);
    }
    if (kmers > 0 && mem_limit > 0 && kmers > mem_limit / 64)
    {
        fprintf(stderr, "Warning: Block size too big, index occupies more than 1/4 of");
        if (mem_physical)
            fprintf(stderr, " physical memory (%.1fGb)\n", (1. * mem_limit) / 0x40000000ll);
        else
            fprintf(stderr, " desired memory allocation (%.1fGb)\n", (1. * mem_limit) / 0x40000000ll);
        fflush(stderr);
    }
}

void gd_report_match(gd_context* ctx, const char* aname, const char* bname, int comp, int same_index, int bslot,
                     int64_t recs_before, double atot, double btot, int kmer, int64_t mem_limit)
{
    gd_stats st;
    gd_get_stats(ctx, &st);
    int64_t tb = 0;
    const int64_t recs = gd_num_overlaps(ctx, &tb);
    const int64_t alen = st.kmers[0], blen = st.kmers[bslot];
    int64_t nhits = 0, nfilt = 0, ncheck = 0;
    if (comp)
        printf("\nComparing %s to c(%s)\n", aname, bname);
    else
        printf("\nComparing %s to %s\n", aname, bname);
    if (alen > 0 && blen > 0)
    {
        printf("\n");
        if (mem_limit > 0)
            printf("   Capping mutual k-mer matches over %d (effectively -t%d)\n", st.limit[comp],
                   (int)sqrt(1. * st.limit[comp]));
        nhits = st.hits[comp];
        printf("   Hit count = ");
        gd_report_number(nhits, 0);
        if (same_index || nhits >= blen)
            printf("\n   Highwater of %.2fGb space\n", (1. * (alen + 2 * nhits)) / 67108864);
        else
            printf("\n   Highwater of %.2fGb space\n", (1. * (alen + blen + nhits)) / 67108864);
        if (nhits > 0)
        {
            nfilt = st.seeds[comp];
            ncheck = recs - recs_before;
        }
    }
    int width = nhits <= 0 ? 1 : (int)log10((double)nhits) + 1;
    width += (width - 1) / 3;
    printf("\n     ");
    gd_report_number(nhits, width);
    printf(" %d-mers (%e of matrix)\n     ", kmer, (1. * nhits / atot) / btot);
    gd_report_number(nfilt, width);
    printf(" seed hits (%e of matrix)\n     ", (1. * nfilt / atot) / btot);
    gd_report_number(ncheck, width);
    printf(" confirmed hits (%e of matrix)\n", (1. * ncheck / atot) / btot);
    fflush(stdout);
}
