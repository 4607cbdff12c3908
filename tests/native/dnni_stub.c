/* A stand-in for libdnni.so with the entry points the nni:: drop-in calls,
 * for CPU tests of the drop-in's host logic (stream reads and seeks).  Each
 * interpolation call appends one line to the file named by DNNI_STUB_LOG:
 * the call, the point count, and the min and max time passed (space-time),
 * and fills the heights with 1. */
#include <stdio.h>
#include <stdlib.h>
#include "dnni.h"

struct dnni_ctx { int unused; };
static struct dnni_ctx g_ctx;

static void log_line(const char *what, int64_t n, int32_t tmin, int32_t tmax) {
    const char *path = getenv("DNNI_STUB_LOG");
    FILE *f = path ? fopen(path, "a") : NULL;
    if (!f) return;
    fprintf(f, "%s %lld %d %d\n", what, (long long)n, (int)tmin, (int)tmax);
    fclose(f);
}

dnni_status dnni_init(const dnni_settings *s, dnni_ctx **out) { (void)s; *out = &g_ctx; return DNNI_OK; }
dnni_status dnni_destroy(dnni_ctx *c) { (void)c; return DNNI_OK; }
const char *dnni_last_error(const dnni_ctx *c) { (void)c; return ""; }
dnni_status dnni_setup_run(dnni_ctx *c, const dnni_workpackage *wp, int64_t m) { (void)c; (void)wp; (void)m; return DNNI_OK; }

dnni_status dnni_interpolate_segment(dnni_ctx *c, const dnni_workpackage *wp, const int32_t *xyz, const uint32_t *gid,
                                     int64_t n, float *h, uint32_t *site, dnni_stats *st) {
    (void)c; (void)xyz; (void)gid; (void)site;
    for (int64_t k = 0; k < (int64_t)wp->ncols * wp->nrows; k++) h[k] = 1.0f;
    if (st) st->ms_total = 0;
    log_line("segment", n, 0, 0);
    return DNNI_OK;
}

dnni_status dnni_interpolate_compat(dnni_ctx *c, const dnni_compat_settings *s, const dnni_compat_wp *wp,
                                    const double *xyz, int64_t n, float *h, int32_t *r) {
    (void)c; (void)s; (void)xyz; (void)r;
    for (int64_t k = 0; k < (int64_t)wp->ncols * wp->nrows; k++) h[k] = 1.0f;
    log_line("compat", n, 0, 0);
    return DNNI_OK;
}

dnni_status dnni_interpolate_spacetime(dnni_ctx *c, const dnni_workpackage *wp, const dnni_st_options *o,
                                       const int32_t *xyz, const int32_t *t, int64_t n, float *h, dnni_stats *st) {
    (void)c; (void)o; (void)xyz;
    int32_t lo = 0, hi = 0;
    for (int64_t k = 0; k < n; k++) {
        if (k == 0 || t[k] < lo) lo = t[k];
        if (k == 0 || t[k] > hi) hi = t[k];
    }
    for (int64_t k = 0; k < (int64_t)wp->ncols * wp->nrows; k++) h[k] = 1.0f;
    if (st) st->ms_total = 0;
    log_line("spacetime", n, lo, hi);
    return DNNI_OK;
}
