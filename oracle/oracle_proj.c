/*
 * CPU oracle for the mbirtorch projector pair -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C with FP64 arithmetic, the separable
 * footprint projectors of mbirtorch (reference v0.0.2).  It exists so that
 * the sm_100a kernels of mbirtorch_b200 can be checked against an independent
 * implementation of the same algorithm.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against golden vectors produced by the reference's own torch bodies
 * (tests/golden/make_golden.py).
 *
 * Layouts follow the reference bodies exactly:
 *   values : (P, L)  voxel cylinders, slice axis contiguous
 *   sino   : (V, R, C) views x detector rows x channels, channel contiguous
 *   out    : (P, L) for back projection
 *
 * Reference formulas followed (file:line in mbirtorch):
 *   tap rule ........... horizontal_fan.py:51-71  (tap_weights)
 *   parallel chain ..... parallel_beam.py:22-53   (_parallel_hfan_math)
 *   parallel fwd/back .. parallel_beam.py:56-94, horizontal_fan.py:74-154
 *   cone chains ........ cone_beam.py:59-158
 *   cone forward ....... cone_beam.py:161-234
 *   cone back .......... cone_beam.py:237-299
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t num_views;          /* views in the arrays passed (a view batch) */
    int32_t num_det_rows;       /* R */
    int32_t num_det_channels;   /* C */
    int32_t num_recon_rows;     /* N rows of the recon grid */
    int32_t num_recon_cols;     /* N cols of the recon grid */
    int32_t num_slices;         /* full slice count S (z anchor) */
    double delta_det_channel;
    double delta_det_row;
    double det_channel_offset;
    double det_row_offset;
    double delta_voxel;
    double delta_voxel_row;
    double delta_voxel_slice;
    double recon_slice_offset;
    double magnification;
    double source_detector_dist;  /* may be +inf */
    int32_t use_curved_detector;
    int32_t psf_radius;
    int32_t bp_psf_radius;
} oracle_geom;

/* Round half to even, like torch.round (default FE_TONEAREST mode). */
static inline long round_half_even(double x) { return (long)nearbyint(x); }

/* horizontal_fan.py:51-71 -- trapezoid weight of channel tap n, zeroed off
 * the detector.  Returns the weight; *n_clamped gets the in-range index. */
static inline double tap_weight(double n_p, long n, double W, double ws,
                                int num_channels, long *n_clamped) {
    double a = (W + 1.0) / 2.0 - fabs(n_p - (double)n);
    if (a < 0.0) a = 0.0;
    double lmax = W < 1.0 ? W : 1.0;
    if (a > lmax) a = lmax;
    a *= ws;
    if (n < 0 || n >= num_channels) a = 0.0;
    long nc = n < 0 ? 0 : (n >= num_channels ? num_channels - 1 : n);
    *n_clamped = nc;
    return a;
}

/* parallel_beam.py:22-53 */
static void parallel_hfan(const oracle_geom *g, double angle, int64_t pixel,
                          double *n_p, long *center, double *W, double *ws) {
    double row = (double)(pixel / g->num_recon_cols);
    double col = (double)(pixel % g->num_recon_cols);
    double y_t = g->delta_voxel_row * (row - (g->num_recon_rows - 1) / 2.0);
    double x_t = g->delta_voxel * (col - (g->num_recon_cols - 1) / 2.0);
    double c = cos(angle), s = sin(angle);
    double x = c * x_t - s * y_t;
    double det_center = (g->num_det_channels - 1) / 2.0;
    *n_p = (x + g->det_channel_offset) / g->delta_det_channel + det_center;
    double fa = fabs(c) * g->delta_voxel, fb = fabs(s) * g->delta_voxel_row;
    double footprint = fa > fb ? fa : fb;
    *W = footprint / g->delta_det_channel;
    *ws = (g->delta_voxel_row * g->delta_voxel) / footprint;
    *center = round_half_even(*n_p);
}

/* Parallel forward: out (V, L, C) = sum_p sum_tap A * values[p, l]
 * (parallel_beam.py:56-73 with horizontal_fan.py:74-107).  Row == slice. */
void oracle_parallel_forward(const oracle_geom *g, const double *angles,
                             const double *values, int32_t L,
                             const int64_t *pixel_indices, int64_t P,
                             double *out) {
    const int V = g->num_views, C = g->num_det_channels, r = g->psf_radius;
    memset(out, 0, sizeof(double) * (size_t)V * L * C);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < V; ++v) {
        double *ov = out + (size_t)v * L * C;
        for (int64_t p = 0; p < P; ++p) {
            double n_p, W, ws;
            long ctr;
            parallel_hfan(g, angles[v], pixel_indices[p], &n_p, &ctr, &W, &ws);
            for (int t = -r; t <= r; ++t) {
                long n;
                double a = tap_weight(n_p, ctr + t, W, ws, C, &n);
                if (a == 0.0) continue;
                const double *vp = values + (size_t)p * L;
                for (int l = 0; l < L; ++l) ov[(size_t)l * C + n] += a * vp[l];
            }
        }
    }
}

/* Parallel back: out (P, L) = sum_v sum_tap A^cp * sino[v, l, c_tap]
 * (parallel_beam.py:76-94 with horizontal_fan.py:110-154). */
void oracle_parallel_back(const oracle_geom *g, const double *angles,
                          const double *sino, int32_t L,
                          const int64_t *pixel_indices, int64_t P,
                          int32_t coeff_power, double *out) {
    const int V = g->num_views, C = g->num_det_channels, r = g->psf_radius;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < P; ++p) {
        double *op = out + (size_t)p * L;
        for (int l = 0; l < L; ++l) op[l] = 0.0;
        for (int v = 0; v < V; ++v) {
            double n_p, W, ws;
            long ctr;
            parallel_hfan(g, angles[v], pixel_indices[p], &n_p, &ctr, &W, &ws);
            const double *sv = sino + (size_t)v * L * C;
            for (int t = -r; t <= r; ++t) {
                long n;
                double a = tap_weight(n_p, ctr + t, W, ws, C, &n);
                if (coeff_power == 2) a = a * a;
                if (a == 0.0) continue;
                for (int l = 0; l < L; ++l) op[l] += a * sv[(size_t)l * C + n];
            }
        }
    }
}

/* Per-(view, pixel) cone quantities: cone_beam.py:59-158. */
typedef struct {
    double n_p, W_c, ws, mag, m0, W_r, z_offset;
    long center;
} cone_vp;

static void cone_geometry(const oracle_geom *g, double angle, double z_shift,
                          int64_t pixel, cone_vp *o) {
    double row = (double)(pixel / g->num_recon_cols);
    double col = (double)(pixel % g->num_recon_cols);
    double y_t = g->delta_voxel_row * (row - (g->num_recon_rows - 1) / 2.0);
    double x_t = g->delta_voxel * (col - (g->num_recon_cols - 1) / 2.0);
    double c = cos(angle), s = sin(angle);
    double x = c * x_t - s * y_t;
    double y = s * x_t + c * y_t;
    double sdd = g->source_detector_dist;
    double mag = 1.0 / (1.0 / g->magnification - y / sdd);
    double u, theta;
    if (!g->use_curved_detector) {
        u = mag * x;
        theta = atan2(u, sdd);
    } else {
        double sid = sdd / g->magnification;
        u = sdd * atan2(x, sid - y);
        theta = u / sdd;
    }
    double det_center = (g->num_det_channels - 1) / 2.0;
    o->n_p = (u + g->det_channel_offset) / g->delta_det_channel + det_center;
    double fa = fabs(cos(angle - theta)) * g->delta_voxel;
    double fb = fabs(sin(angle - theta)) * g->delta_voxel_row;
    double footprint = fa > fb ? fa : fb;
    if (!g->use_curved_detector)
        o->W_c = mag * (footprint / g->delta_det_channel) / cos(theta);
    else
        o->W_c = mag * (footprint / g->delta_det_channel);
    o->ws = (g->delta_voxel_row * g->delta_voxel) / footprint;
    o->center = round_half_even(o->n_p);
    o->mag = mag;
    /* _cone_vertical_affine */
    o->z_offset = g->recon_slice_offset - z_shift;
    double det_center_row = (g->num_det_rows - 1) / 2.0;
    o->W_r = mag * g->delta_voxel_slice / g->delta_det_row;
    double z0 = o->z_offset - g->delta_voxel_slice * (g->num_slices - 1) / 2.0;
    o->m0 = (mag * z0 + g->det_row_offset) / g->delta_det_row + det_center_row;
}

static inline double cone_cos_phi(const oracle_geom *g, const cone_vp *q,
                                  double k_global) {
    double z = g->delta_voxel_slice * (k_global - (g->num_slices - 1) / 2.0)
               + q->z_offset;
    return cos(atan2(q->mag * z, g->source_detector_dist));
}

/* Cone forward (cone_beam.py:161-234): detector-side vertical fan with
 * bp_psf_radius slice taps, then the horizontal scatter.  values is a slice
 * band (P, L) starting at global slice slice_start.  out (V, R, C). */
void oracle_cone_forward(const oracle_geom *g, const double *view_params,
                         const double *values, int32_t L, int32_t slice_start,
                         const int64_t *pixel_indices, int64_t P, double *out) {
    const int V = g->num_views, C = g->num_det_channels, R = g->num_det_rows;
    const int r = g->psf_radius, bp = g->bp_psf_radius;
    memset(out, 0, sizeof(double) * (size_t)V * R * C);
#pragma omp parallel
    {
        double *det_col = (double *)malloc(sizeof(double) * (size_t)R);
        double *scaled = (double *)malloc(sizeof(double) * (size_t)(L > 0 ? L : 1));
#pragma omp for schedule(static)
        for (int v = 0; v < V; ++v) {
            double *ov = out + (size_t)v * R * C;
            for (int64_t p = 0; p < P; ++p) {
                cone_vp q;
                cone_geometry(g, view_params[2 * v], view_params[2 * v + 1],
                              pixel_indices[p], &q);
                const double *vp = values + (size_t)p * L;
                for (int l = 0; l < L; ++l)
                    scaled[l] = vp[l] / cone_cos_phi(g, &q, (double)(slice_start + l));
                double slope = q.W_r;
                double lmax = slope < 1.0 ? slope : 1.0;
                for (int m = 0; m < R; ++m) {
                    double k_m = ((double)m - q.m0) / slope;
                    long kc = round_half_even(k_m);
                    double m_p = slope * ((double)kc - k_m);
                    double acc = 0.0;
                    for (int ko = -bp; ko <= bp; ++ko) {
                        long k_ind = kc + ko;
                        double a = (slope + 1.0) / 2.0 - fabs(m_p + slope * ko);
                        if (a < 0.0) a = 0.0;
                        if (a > lmax) a = lmax;
                        if (k_ind < slice_start || k_ind >= slice_start + L) continue;
                        acc += a * scaled[k_ind - slice_start];
                    }
                    det_col[m] = acc;
                }
                for (int t = -r; t <= r; ++t) {
                    long n;
                    double a = tap_weight(q.n_p, q.center + t, q.W_c, q.ws, C, &n);
                    if (a == 0.0) continue;
                    for (int m = 0; m < R; ++m) ov[(size_t)m * C + n] += a * det_col[m];
                }
            }
        }
        free(det_col);
        free(scaled);
    }
}

/* Cone back (cone_beam.py:237-299): horizontal gather per view into detector
 * columns, then the vertical gather onto the band [slice_start,
 * slice_start + band) with psf_radius row taps.  out (P, band). */
void oracle_cone_back(const oracle_geom *g, const double *view_params,
                      const double *sino, int32_t coeff_power,
                      int32_t slice_start, int32_t band,
                      const int64_t *pixel_indices, int64_t P, double *out) {
    const int V = g->num_views, C = g->num_det_channels, R = g->num_det_rows;
    const int r = g->psf_radius;
#pragma omp parallel
    {
        double *det_col = (double *)malloc(sizeof(double) * (size_t)R);
#pragma omp for schedule(static)
        for (int64_t p = 0; p < P; ++p) {
            double *op = out + (size_t)p * band;
            for (int l = 0; l < band; ++l) op[l] = 0.0;
            for (int v = 0; v < V; ++v) {
                cone_vp q;
                cone_geometry(g, view_params[2 * v], view_params[2 * v + 1],
                              pixel_indices[p], &q);
                const double *sv = sino + (size_t)v * R * C;
                for (int m = 0; m < R; ++m) det_col[m] = 0.0;
                for (int t = -r; t <= r; ++t) {
                    long n;
                    double a = tap_weight(q.n_p, q.center + t, q.W_c, q.ws, C, &n);
                    if (coeff_power == 2) a = a * a;
                    if (a == 0.0) continue;
                    for (int m = 0; m < R; ++m) det_col[m] += a * sv[(size_t)m * C + n];
                }
                double slope = q.W_r;
                double lmax = slope < 1.0 ? slope : 1.0;
                for (int l = 0; l < band; ++l) {
                    double k = (double)(slice_start + l);
                    double cos_phi = cone_cos_phi(g, &q, k);
                    double m_p = q.m0 + slope * k;
                    long mc = round_half_even(m_p);
                    double acc = 0.0;
                    for (int t = -r; t <= r; ++t) {
                        long mm = mc + t;
                        double a = (slope + 1.0) / 2.0 - fabs(m_p - (double)mm);
                        if (a < 0.0) a = 0.0;
                        if (a > lmax) a = lmax;
                        a = a / cos_phi;
                        if (mm < 0 || mm >= R) a = 0.0;
                        if (coeff_power == 2) a = a * a;
                        if (a == 0.0) continue;
                        acc += a * det_col[mm];
                    }
                    op[l] += acc;
                }
            }
        }
        free(det_col);
    }
}
