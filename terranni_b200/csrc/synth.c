/*
 * synth.c -- seeded synthetic LiDAR-like point clouds for the NNI engine's
 * benchmarks and tests (host code, OpenMP).
 *
 * The reference's only data source is a Python 2 text generator
 * (data-generator.py:49-100: uniform xy on [-100,100]^2, random z) whose output
 * no reference reader consumes; the workloads here are the ones the benchmark
 * configurations name instead:
 *   kind 1  "sinusoid": x,y uniform over the extent, z = sum of 4 directional
 *           sinusoids (amplitude 5-20 m, wavelength 30-200 m, seeded phases)
 *           plus N(0, z_noise);
 *   kind 0  "terrain": a fraction of points uniform, the rest in Gaussian
 *           clusters, circular "lakes" with no points inside, z = value-noise
 *           fBm (Hurst H, `octaves` octaves) rescaled to [0, relief] plus
 *           N(0, z_noise).
 * Coordinates are written as int32 LAS units: X = llround(x / xy_scale) with
 * x measured from the extent's origin, likewise Z = llround(z / z_scale).
 *
 * Every point draws from its own counter-based stream (splitmix64 of the seed
 * and the point index), so the output does not depend on the thread count.
 */
#include <stdint.h>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    uint64_t seed;
    int64_t n;
    double width, height;          /* extent in metres, origin at (0,0) */
    double xy_scale, z_scale;      /* metres per LAS unit */
    int32_t kind;                  /* 0 terrain, 1 sinusoid */
    int32_t nclusters;
    double frac_uniform;
    double cluster_sigma;
    int32_t nlakes;
    int32_t octaves;
    double lake_rmin, lake_rmax;
    double relief, z_noise, hurst, base_wavelength;
    int32_t nthreads;              /* 0 = OpenMP default */
    int32_t pad;
} synth_params;

static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct { uint64_t s; } rng_t;

static inline uint64_t rng_next(rng_t *r) { r->s += 0x9E3779B97F4A7C15ull; return mix64(r->s); }
static inline double rng_u01(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline double rng_normal(rng_t *r) {
    double u1 = rng_u01(r), u2 = rng_u01(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* value noise: hashed lattice values in [-1,1], quintic interpolation */
static inline double lattice(uint64_t seed, int64_t ix, int64_t iy, int oct) {
    uint64_t h = mix64(seed ^ mix64((uint64_t)ix * 0x9E3779B97F4A7C15ull ^ mix64((uint64_t)iy + 0x632BE59BD9B4E019ull * (uint64_t)(oct + 1))));
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static inline double fade(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }

static double value_noise(uint64_t seed, double x, double y, int oct) {
    double fx = floor(x), fy = floor(y);
    int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    double tx = fade(x - fx), ty = fade(y - fy);
    double v00 = lattice(seed, ix, iy, oct), v10 = lattice(seed, ix + 1, iy, oct);
    double v01 = lattice(seed, ix, iy + 1, oct), v11 = lattice(seed, ix + 1, iy + 1, oct);
    double a = v00 + (v10 - v00) * tx, b = v01 + (v11 - v01) * tx;
    return a + (b - a) * ty;
}

static double fbm(const synth_params *p, double x, double y) {
    double v = 0.0, amp = 1.0, f = 1.0 / p->base_wavelength;
    double decay = pow(2.0, -p->hurst);
    for (int o = 0; o < p->octaves; o++) {
        v += amp * value_noise(p->seed, x * f, y * f, o);
        amp *= decay;
        f *= 2.0;
    }
    return v;
}

typedef struct { double A, kx, ky, phi; } sinus_t;

/* Fills lakes (nlakes x 3: cx, cy, r metres) and clusters (nclusters x 2)
 * from the seed; exposed so that callers can report the realised layout. */
int synth_layout(const synth_params *p, double *lakes, double *clusters) {
    rng_t r = { mix64(p->seed ^ 0x5EEDF00Dull) };
    for (int i = 0; i < p->nlakes; i++) {
        double rad = p->lake_rmin + (p->lake_rmax - p->lake_rmin) * rng_u01(&r);
        lakes[3 * i + 0] = rng_u01(&r) * p->width;
        lakes[3 * i + 1] = rng_u01(&r) * p->height;
        lakes[3 * i + 2] = rad;
    }
    for (int i = 0; i < p->nclusters; i++) {
        clusters[2 * i + 0] = rng_u01(&r) * p->width;
        clusters[2 * i + 1] = rng_u01(&r) * p->height;
    }
    return 0;
}

/* Uniform grid over the area listing the lakes whose bounding box meets each
 * grid cell (CSR), so that a point is tested only against the lakes near it;
 * a point is in a lake when it is strictly inside any lake's circle. */
typedef struct {
    int g;            /* cells per side */
    double cw, ch;    /* cell size */
    int *start, *ids;
} lake_grid;

static void lake_grid_build(lake_grid *lg, const double *lakes, int nl, double width, double height) {
    int g = (int)ceil(sqrt((double)nl));
    if (g < 1) g = 1;
    if (g > 1024) g = 1024;
    lg->g = g;
    lg->cw = width / g;
    lg->ch = height / g;
    lg->start = (int *)calloc((size_t)g * g + 1, sizeof(int));
    for (int pass = 0; pass < 2; pass++) {
        int *fill = pass ? (int *)calloc((size_t)g * g, sizeof(int)) : NULL;
        for (int i = 0; i < nl; i++) {
            double r = lakes[3 * i + 2];
            int x0 = (int)floor((lakes[3 * i] - r) / lg->cw), x1 = (int)floor((lakes[3 * i] + r) / lg->cw);
            int y0 = (int)floor((lakes[3 * i + 1] - r) / lg->ch), y1 = (int)floor((lakes[3 * i + 1] + r) / lg->ch);
            if (x0 < 0) x0 = 0;
            if (y0 < 0) y0 = 0;
            if (x1 > g - 1) x1 = g - 1;
            if (y1 > g - 1) y1 = g - 1;
            for (int y = y0; y <= y1; y++)
                for (int x = x0; x <= x1; x++) {
                    if (pass == 0) lg->start[y * g + x + 1]++;
                    else lg->ids[lg->start[y * g + x] + fill[y * g + x]++] = i;
                }
        }
        if (pass == 0) {
            for (int k = 0; k < g * g; k++) lg->start[k + 1] += lg->start[k];
            lg->ids = (int *)malloc(sizeof(int) * (size_t)(lg->start[g * g] > 0 ? lg->start[g * g] : 1));
        } else {
            free(fill);
        }
    }
}

static inline int in_lake_grid(const lake_grid *lg, const double *lakes, double x, double y) {
    int cx = (int)(x / lg->cw), cy = (int)(y / lg->ch);
    if (cx < 0) cx = 0;
    if (cy < 0) cy = 0;
    if (cx > lg->g - 1) cx = lg->g - 1;
    if (cy > lg->g - 1) cy = lg->g - 1;
    const int c = cy * lg->g + cx;
    for (int k = lg->start[c]; k < lg->start[c + 1]; k++) {
        const int i = lg->ids[k];
        double dx = x - lakes[3 * i], dy = y - lakes[3 * i + 1];
        if (dx * dx + dy * dy < lakes[3 * i + 2] * lakes[3 * i + 2]) return 1;
    }
    return 0;
}

/* Generates p->n points into xyz (n x 3 int32).  Returns 0, or 1 on bad
 * parameters.  lakes_out (nlakes x 3) may be NULL. */
int synth_generate(const synth_params *p, int32_t *xyz, double *lakes_out) {
    if (p->n < 0 || p->width <= 0 || p->height <= 0 || p->xy_scale <= 0 || p->z_scale <= 0) return 1;
    int nl = p->kind == 0 ? p->nlakes : 0;
    int ncl = p->kind == 0 ? p->nclusters : 0;
    double *lakes = (double *)calloc((size_t)(nl > 0 ? nl : 1) * 3, sizeof(double));
    double *clus = (double *)calloc((size_t)(ncl > 0 ? ncl : 1) * 2, sizeof(double));
    synth_params q = *p;
    q.nlakes = nl; q.nclusters = ncl;
    synth_layout(&q, lakes, clus);
    if (lakes_out && nl) memcpy(lakes_out, lakes, sizeof(double) * 3 * (size_t)nl);

    /* fBm range over a coarse lattice, for the [0, relief] rescale */
    double vmin = 1e300, vmax = -1e300;
    if (p->kind == 0) {
        for (int j = 0; j <= 128; j++)
            for (int i = 0; i <= 128; i++) {
                double v = fbm(p, p->width * i / 128.0, p->height * j / 128.0);
                if (v < vmin) vmin = v;
                if (v > vmax) vmax = v;
            }
        if (vmax - vmin < 1e-12) vmax = vmin + 1.0;
    }
    sinus_t sn[4];
    {
        rng_t r = { mix64(p->seed ^ 0xABCDEF12345ull) };
        for (int k = 0; k < 4; k++) {
            double A = 5.0 + 15.0 * rng_u01(&r);
            double lam = 30.0 + 170.0 * rng_u01(&r);
            double th = 6.283185307179586 * rng_u01(&r);
            sn[k].A = A;
            sn[k].kx = cos(th) * 6.283185307179586 / lam;
            sn[k].ky = sin(th) * 6.283185307179586 / lam;
            sn[k].phi = 6.283185307179586 * rng_u01(&r);
        }
    }
    lake_grid lg;
    lake_grid_build(&lg, lakes, nl, p->width, p->height);
    int64_t n = p->n;
    int64_t xmax_u = (int64_t)floor(p->width / p->xy_scale), ymax_u = (int64_t)floor(p->height / p->xy_scale);
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        rng_t r = { mix64(p->seed * 0x2545F4914F6CDD1Dull ^ mix64((uint64_t)i)) };
        double x = 0, y = 0;
        for (int attempt = 0; attempt < 100000; attempt++) {
            if (ncl == 0 || rng_u01(&r) < p->frac_uniform) {
                x = rng_u01(&r) * p->width;
                y = rng_u01(&r) * p->height;
            } else {
                int c = (int)(rng_u01(&r) * ncl);
                if (c >= ncl) c = ncl - 1;
                x = clus[2 * c] + p->cluster_sigma * rng_normal(&r);
                y = clus[2 * c + 1] + p->cluster_sigma * rng_normal(&r);
                if (x < 0 || y < 0 || x >= p->width || y >= p->height) continue;
            }
            if (!in_lake_grid(&lg, lakes, x, y)) break;
        }
        double z;
        if (p->kind == 1) {
            z = 0;
            for (int k = 0; k < 4; k++) z += sn[k].A * sin(sn[k].kx * x + sn[k].ky * y + sn[k].phi);
        } else {
            z = (fbm(p, x, y) - vmin) / (vmax - vmin) * p->relief;
        }
        z += p->z_noise * rng_normal(&r);
        int64_t X = llround(x / p->xy_scale), Y = llround(y / p->xy_scale);
        if (X > xmax_u - 1) X = xmax_u - 1;
        if (Y > ymax_u - 1) Y = ymax_u - 1;
        if (X < 0) X = 0;
        if (Y < 0) Y = 0;
        xyz[3 * i + 0] = (int32_t)X;
        xyz[3 * i + 1] = (int32_t)Y;
        xyz[3 * i + 2] = (int32_t)llround(z / p->z_scale);
    }
    free(lg.start); free(lg.ids);
    free(lakes); free(clus);
    return 0;
}
