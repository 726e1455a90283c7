/*
 * CPU oracle for the six-band listener-space path tracer.  TEST
 * INFRASTRUCTURE ONLY: the parity tests, the smoke check and the CPU
 * baseline leg of the benchmark call it as the checker.  Nothing in the
 * product links against it.
 *
 * This is a scalar float64 restatement of Acoustic Agent's Numba tracer,
 * written to reproduce its arithmetic operation by operation:
 *   - acoustic_agent/steam_rt.py:4259-4274  _point_in_polygon_jit
 *   - acoustic_agent/steam_rt.py:4277-4358  _box_hit_jit
 *   - acoustic_agent/steam_rt.py:4361-4392  _surface_hit_jit
 *   - acoustic_agent/steam_rt.py:4406-4426  _ray_aabb_intersects_jit
 *   - acoustic_agent/steam_rt.py:4429-4478  _closest_hit_jit (linear)
 *   - acoustic_agent/steam_rt.py:4481-4506  _closest_hit_bvh_jit (escape walk)
 *   - acoustic_agent/steam_rt.py:4522-4533  _ray_sphere_before_jit
 *   - acoustic_agent/steam_rt.py:4556-4582  _normalize3_jit, _diffuse_direction_jit
 *   - acoustic_agent/steam_rt.py:4708-4850  _trace_energy_kernel body
 *   - acoustic_agent/steam_rt.py:4131-4146  _biquad_filter_jit
 *   - acoustic_agent/steam_rt.py:2205-2232  reconstruct_band_irs envelope
 *   - acoustic_agent/steam_rt.py:3070-3083  bandlimit_band_signals
 *   - acoustic_agent/steam_rt.py:2235-2327  _fdn_impulse_kernel (16-line FDN)
 *
 * Build with -ffp-contract=off and without -ffast-math: Numba evaluates
 * every multiply and add separately in IEEE double, and so must this file.
 * libm pow/sqrt/floor are the same functions Numba's LLVM calls resolve to.
 *
 * Beyond the reference outputs, the oracle records per-ray hit-surface
 * sequences and counts BVH nodes / primitives visited in the reference's
 * traversal order; the benchmark turns those counts into algorithmic bytes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NB 6
static const double EPS = 1e-6;           /* steam_rt.py:37 _EPS */
static const double HIT_OFFSET = 1e-2;    /* steam_rt.py:41 _HIT_OFFSET */
static const double BVH_EPS = 2.0e-6;     /* steam_rt.py:44 _BVH_BOUNDS_EPS */
static const double PI = 3.141592653589793;

typedef struct {
    int64_t num_surfaces;
    const int64_t *kinds;        /* [S] 0 wall, 1 horizontal polygon, 2 box */
    const double *wall_a;        /* [S,2] */
    const double *wall_delta;    /* [S,2] */
    const double *wall_z;        /* [S,2] */
    const double *z_values;      /* [S] */
    const double *box_center;    /* [S,2] */
    const double *box_axis_u;    /* [S,2] */
    const double *box_axis_v;    /* [S,2] */
    const double *box_half;      /* [S,2] */
    const double *box_z;         /* [S,2] */
    const double *normals;       /* [S,3] */
    const double *reflection;    /* [S,6] */
    const double *scattering;    /* [S] */
    int64_t num_corners;
    const double *corners;       /* [C,2] */
    int64_t num_nodes;
    const double *bvh_min;       /* [N,3] */
    const double *bvh_max;       /* [N,3] */
    const int64_t *bvh_start;    /* [N] */
    const int64_t *bvh_count;    /* [N] */
    const int64_t *bvh_escape;   /* [N] */
    const int64_t *bvh_prims;    /* [P] */
    int64_t use_bvh;
} oracle_scene;

typedef struct {
    double source[3];
    double listener[3];
    double source_forward[3];
    int64_t num_rays;
    int64_t num_bounces;
    int64_t num_bins;
    int64_t num_bank;
    double bin_dur;
    double c;
    double max_path_len;
    double direct_delay;
    double listener_radius;
    double source_radius;
    double irradiance_min_distance;
    double specular_exponent;
    double dipole_weight;
    double dipole_power;
    int64_t render_ambisonics;
    int64_t num_threads;         /* <= 0: all available */
    const double *directions;    /* [R,3] */
    const double *diffuse_bank;  /* [K,3] */
    const double *diffuse_random;/* [B,R] */
    const int32_t *diffuse_indices; /* [B,R] */
} oracle_params;

typedef struct {
    double *echogram;            /* [6,bins] */
    double *ambisonic;           /* [6,4,bins] or NULL */
    int64_t *hit_counts;         /* [S] */
    int64_t *contrib_counts;     /* [S] */
    double *surface_energy;      /* [S] */
    int64_t actual_bounces;
    int64_t active_count;
    int32_t *ray_surfaces;       /* [R,B] or NULL: hit surface per bounce, -1 after termination */
    int32_t *ray_bounces;        /* [R] or NULL: closest-hit queries issued per ray */
    /* traversal statistics in the reference's visiting order */
    int64_t closest_queries;
    int64_t shadow_queries;
    int64_t nodes_visited;
    int64_t prims_tested[3];
    int64_t polygon_edges;
    /* [R,B,7] or NULL: the ray's state before each closest-hit query (origin xyz, direction xyz, path
     * length so far), NaN once the ray has ended; for locating where a float32 trace parts from this one */
    double *ray_states;
} oracle_outputs;

typedef struct {
    int64_t nodes;
    int64_t prims[3];
    int64_t edges;
} visit_stats;

static int point_in_polygon(double x, double y, const double *corners, int64_t n, visit_stats *st)
{
    int inside = 0;
    int64_t j = n - 1;
    for (int64_t i = 0; i < n; ++i) {
        double xi = corners[2 * i], yi = corners[2 * i + 1];
        double xj = corners[2 * j], yj = corners[2 * j + 1];
        if ((yi > y) != (yj > y)) {
            double denom = yj - yi;
            if (fabs(denom) > 1e-12) {
                double x_cross = (xj - xi) * (y - yi) / denom + xi;
                if (x < x_cross) inside = !inside;
            }
        }
        j = i;
    }
    st->edges += n;
    return inside;
}

/* steam_rt.py:4277-4358; returns t (1e30 on miss) and the entry/exit normal. */
static double box_hit(const double *o, const double *d, const double *center, const double *au,
                      const double *av, const double *half, const double *zr, double *n)
{
    double relx = o[0] - center[0];
    double rely = o[1] - center[1];
    double ox = relx * au[0] + rely * au[1];
    double oy = relx * av[0] + rely * av[1];
    double oz = o[2];
    double dx = d[0] * au[0] + d[1] * au[1];
    double dy = d[0] * av[0] + d[1] * av[1];
    double dz = d[2];
    double t_min = -1.0e30, t_max = 1.0e30;
    double nx = 0.0, ny = 0.0, nz = 0.0, ex = 0.0, ey = 0.0, ez = 0.0;
    for (int axis = 0; axis < 3; ++axis) {
        double oo, dd, lo, hi, ax, ay, az;
        if (axis == 0) { oo = ox; dd = dx; lo = -half[0]; hi = half[0]; ax = au[0]; ay = au[1]; az = 0.0; }
        else if (axis == 1) { oo = oy; dd = dy; lo = -half[1]; hi = half[1]; ax = av[0]; ay = av[1]; az = 0.0; }
        else { oo = oz; dd = dz; lo = zr[0]; hi = zr[1]; ax = 0.0; ay = 0.0; az = 1.0; }
        if (fabs(dd) <= 1.0e-12) {
            if (oo < lo || oo > hi) { n[0] = 0.0; n[1] = 0.0; n[2] = 1.0; return 1.0e30; }
            continue;
        }
        double enter, exit_, enx, eny, enz, oux, ouy, ouz;
        if (dd > 0.0) {
            enter = (lo - oo) / dd; exit_ = (hi - oo) / dd;
            enx = -ax; eny = -ay; enz = -az; oux = ax; ouy = ay; ouz = az;
        } else {
            enter = (hi - oo) / dd; exit_ = (lo - oo) / dd;
            enx = ax; eny = ay; enz = az; oux = -ax; ouy = -ay; ouz = -az;
        }
        if (enter > t_min) { t_min = enter; nx = enx; ny = eny; nz = enz; }
        if (exit_ < t_max) { t_max = exit_; ex = oux; ey = ouy; ez = ouz; }
        if (t_min > t_max) { n[0] = 0.0; n[1] = 0.0; n[2] = 1.0; return 1.0e30; }
    }
    if (t_max <= EPS) { n[0] = 0.0; n[1] = 0.0; n[2] = 1.0; return 1.0e30; }
    if (t_min > EPS) { n[0] = nx; n[1] = ny; n[2] = nz; return t_min; }
    n[0] = ex; n[1] = ey; n[2] = ez;
    return t_max;
}

/* steam_rt.py:4361-4392 */
static double surface_hit(const oracle_scene *sc, int64_t si, const double *o, const double *d, double *n,
                          visit_stats *st)
{
    double t = 1e30;
    n[0] = sc->normals[3 * si]; n[1] = sc->normals[3 * si + 1]; n[2] = sc->normals[3 * si + 2];
    int64_t kind = sc->kinds[si];
    if (kind == 0) {
        st->prims[0] += 1;
        double sx = sc->wall_delta[2 * si], sy = sc->wall_delta[2 * si + 1];
        double det = sx * d[1] - sy * d[0];
        if (fabs(det) > 1e-12) {
            double relx = o[0] - sc->wall_a[2 * si];
            double rely = o[1] - sc->wall_a[2 * si + 1];
            double cand_t = (relx * sy - rely * sx) / det;
            double u = (relx * d[1] - rely * d[0]) / det;
            double z = o[2] + cand_t * d[2];
            if (cand_t > EPS && u >= -1e-6 && u <= 1.0 + 1e-6 && z >= sc->wall_z[2 * si] - 1e-6 &&
                z <= sc->wall_z[2 * si + 1] + 1e-6)
                t = cand_t;
        }
    } else if (kind == 2) {
        st->prims[2] += 1;
        double bn[3];
        double cand_t = box_hit(o, d, sc->box_center + 2 * si, sc->box_axis_u + 2 * si, sc->box_axis_v + 2 * si,
                                sc->box_half + 2 * si, sc->box_z + 2 * si, bn);
        if (cand_t > EPS && cand_t < 1.0e29) {
            t = cand_t; n[0] = bn[0]; n[1] = bn[1]; n[2] = bn[2];
        }
    } else {
        st->prims[1] += 1;
        if (fabs(d[2]) > 1e-12) {
            double cand_t = (sc->z_values[si] - o[2]) / d[2];
            double px = o[0] + cand_t * d[0];
            double py = o[1] + cand_t * d[1];
            if (cand_t > EPS && point_in_polygon(px, py, sc->corners, sc->num_corners, st)) t = cand_t;
        }
    }
    return t;
}

/* steam_rt.py:4406-4426 */
static int ray_aabb(const double *o, const double *d, const double *lo, const double *hi, double max_distance)
{
    double enter = 0.0;
    double exit_ = max_distance + BVH_EPS;
    for (int axis = 0; axis < 3; ++axis) {
        double value = d[axis];
        if (fabs(value) <= 1e-15) {
            if (o[axis] < lo[axis] || o[axis] > hi[axis]) return 0;
            continue;
        }
        double first = (lo[axis] - o[axis]) / value;
        double second = (hi[axis] - o[axis]) / value;
        if (first > second) { double tmp = first; first = second; second = tmp; }
        if (first > enter) enter = first;
        if (second < exit_) exit_ = second;
        if (enter > exit_) return 0;
    }
    return exit_ > EPS;
}

/* steam_rt.py:4429-4506: linear scan or escape-link BVH walk; normal oriented against the ray. */
static int64_t closest_hit(const oracle_scene *sc, const double *o, const double *d, double *t_out, double *n_out,
                           visit_stats *st)
{
    double best_t = 1e30;
    int64_t best = -1;
    double bn[3] = {0.0, 0.0, 0.0};
    double n[3];
    if (sc->use_bvh) {
        int64_t node = 0;
        while (node < sc->num_nodes) {
            st->nodes += 1;
            if (!ray_aabb(o, d, sc->bvh_min + 3 * node, sc->bvh_max + 3 * node, best_t)) {
                node = sc->bvh_escape[node];
                continue;
            }
            int64_t count = sc->bvh_count[node];
            if (count > 0) {
                int64_t start = sc->bvh_start[node];
                for (int64_t k = 0; k < count; ++k) {
                    int64_t si = sc->bvh_prims[start + k];
                    double t = surface_hit(sc, si, o, d, n, st);
                    /* A miss (t == 1e30) still wins while best_surface < 0: the
                     * reference's tie rule, kept so escaped rays count the same. */
                    if (t < best_t || (t == best_t && (best < 0 || si < best))) {
                        best_t = t; best = si; bn[0] = n[0]; bn[1] = n[1]; bn[2] = n[2];
                    }
                }
            }
            node += 1;
        }
    } else {
        for (int64_t si = 0; si < sc->num_surfaces; ++si) {
            double t = surface_hit(sc, si, o, d, n, st);
            if (t < best_t) { best_t = t; best = si; bn[0] = n[0]; bn[1] = n[1]; bn[2] = n[2]; }
        }
    }
    if (best >= 0) {
        double dot = bn[0] * d[0] + bn[1] * d[1] + bn[2] * d[2];
        if (dot > 0.0) { bn[0] = -bn[0]; bn[1] = -bn[1]; bn[2] = -bn[2]; }
    }
    *t_out = best_t;
    n_out[0] = bn[0]; n_out[1] = bn[1]; n_out[2] = bn[2];
    return best;
}

static int sphere_before(const double *o, const double *d, double cx, double cy, double cz, double radius,
                         double max_distance)
{
    double ox = o[0] - cx, oy = o[1] - cy, oz = o[2] - cz;
    double b = ox * d[0] + oy * d[1] + oz * d[2];
    double c = ox * ox + oy * oy + oz * oz - radius * radius;
    double disc = b * b - c;
    if (disc < 0.0) return 0;
    double root = -b - sqrt(disc > 0.0 ? disc : 0.0);
    return root >= 0.0 && root < max_distance;
}

static void normalize3(double x, double y, double z, double *out)
{
    double n = sqrt(x * x + y * y + z * z);
    if (n <= 1e-12) { out[0] = 0.0; out[1] = 0.0; out[2] = 0.0; return; }
    out[0] = x / n; out[1] = y / n; out[2] = z / n;
}

static void diffuse_direction(const double *s, double nx, double ny, double nz, double *out)
{
    double hx = 1.0, hy = 0.0, hz = 0.0;
    if (fabs(nx) >= 0.9) { hx = 0.0; hy = 1.0; }
    double t[3];
    normalize3(hy * nz - hz * ny, hz * nx - hx * nz, hx * ny - hy * nx, t);
    double bx = ny * t[2] - nz * t[1];
    double by = nz * t[0] - nx * t[2];
    double bz = nx * t[1] - ny * t[0];
    normalize3(s[0] * t[0] + s[1] * bx + s[2] * nx, s[0] * t[1] + s[1] * by + s[2] * ny,
               s[0] * t[2] + s[1] * bz + s[2] * nz, out);
}

int oracle_closest_hit(const oracle_scene *sc, const double *origin, const double *direction, double *t_out,
                       double *normal_out)
{
    visit_stats st;
    memset(&st, 0, sizeof(st));
    return (int)closest_hit(sc, origin, direction, t_out, normal_out, &st);
}

int oracle_trace(const oracle_scene *sc, const oracle_params *p, oracle_outputs *out)
{
    const int64_t S = sc->num_surfaces, R = p->num_rays, B = p->num_bounces, NBIN = p->num_bins;
    if (S < 1 || R < 1 || B < 0 || NBIN < 1) return -1;
    int threads = 1;
#ifdef _OPENMP
    threads = p->num_threads > 0 ? (int)p->num_threads : omp_get_max_threads();
#endif
    const int amb = p->render_ambisonics && out->ambisonic != NULL;
    double *l_echo = calloc((size_t)threads * NB * NBIN, sizeof(double));
    double *l_amb = amb ? calloc((size_t)threads * NB * 4 * NBIN, sizeof(double)) : NULL;
    int64_t *l_hits = calloc((size_t)threads * S, sizeof(int64_t));
    int64_t *l_contrib = calloc((size_t)threads * S, sizeof(int64_t));
    double *l_energy = calloc((size_t)threads * S, sizeof(double));
    int64_t *l_active = calloc((size_t)threads, sizeof(int64_t));
    int64_t *l_bounces = calloc((size_t)threads, sizeof(int64_t));
    visit_stats *l_stats = calloc((size_t)threads, sizeof(visit_stats));
    int64_t *l_closest = calloc((size_t)threads, sizeof(int64_t));
    int64_t *l_shadow = calloc((size_t)threads, sizeof(int64_t));
    if (!l_echo || (amb && !l_amb) || !l_hits || !l_contrib || !l_energy || !l_active || !l_bounces || !l_stats ||
        !l_closest || !l_shadow) {
        free(l_echo); free(l_amb); free(l_hits); free(l_contrib); free(l_energy); free(l_active);
        free(l_bounces); free(l_stats); free(l_closest); free(l_shadow);
        return -2;
    }
    const double *src = p->source, *lst = p->listener, *fwd = p->source_forward;
    const double ray_scale = (4.0 * PI) / (double)(R > 1 ? R : 1);

#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t ri = 0; ri < R; ++ri) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *echo = l_echo + (size_t)tid * NB * NBIN;
        double *ambi = amb ? l_amb + (size_t)tid * NB * 4 * NBIN : NULL;
        visit_stats *st = l_stats + tid;
        double origin[3] = {lst[0], lst[1], lst[2]};
        double dir[3] = {p->directions[3 * ri], p->directions[3 * ri + 1], p->directions[3 * ri + 2]};
        double acc[NB] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
        double accum_distance = 0.0;
        int alive = 1;
        int32_t queries = 0;
        if (out->ray_surfaces)
            for (int64_t b = 0; b < B; ++b) out->ray_surfaces[ri * B + b] = -1;
        if (out->ray_states)
            for (int64_t k = 0; k < B * 7; ++k) out->ray_states[ri * B * 7 + k] = NAN;
        for (int64_t bounce = 0; bounce < B; ++bounce) {
            if (bounce + 1 > l_bounces[tid]) l_bounces[tid] = bounce + 1;
            if (out->ray_states) {
                double *rs = out->ray_states + (ri * B + bounce) * 7;
                rs[0] = origin[0]; rs[1] = origin[1]; rs[2] = origin[2];
                rs[3] = dir[0]; rs[4] = dir[1]; rs[5] = dir[2]; rs[6] = accum_distance;
            }
            double t, n[3];
            int64_t surf = closest_hit(sc, origin, dir, &t, n, st);
            l_closest[tid] += 1;
            queries += 1;
            if (surf < 0 || t <= p->listener_radius || accum_distance > p->max_path_len) { alive = 0; break; }
            if (bounce > 0) {
                if (sphere_before(origin, dir, lst[0], lst[1], lst[2], p->listener_radius, t)) { alive = 0; break; }
                double dx = lst[0] - src[0], dy = lst[1] - src[1], dz = lst[2] - src[2];
                double source_distance = sqrt(dx * dx + dy * dy + dz * dz);
                if (source_distance > p->source_radius &&
                    sphere_before(origin, dir, src[0], src[1], src[2], p->source_radius, t)) { alive = 0; break; }
            }
            l_hits[(size_t)tid * S + surf] += 1;
            if (out->ray_surfaces) out->ray_surfaces[ri * B + bounce] = (int32_t)surf;
            double hx = origin[0] + t * dir[0] + HIT_OFFSET * n[0];
            double hy = origin[1] + t * dir[1] + HIT_OFFSET * n[1];
            double hz = origin[2] + t * dir[2] + HIT_OFFSET * n[2];
            double tsx = src[0] - hx, tsy = src[1] - hy, tsz = src[2] - hz;
            double dist = sqrt(tsx * tsx + tsy * tsy + tsz * tsz);
            if (dist > p->irradiance_min_distance) {
                double sdx = tsx / dist, sdy = tsy / dist, sdz = tsz / dist;
                double facing = n[0] * sdx + n[1] * sdy + n[2] * sdz;
                if (facing > 0.0) {
                    double so[3] = {hx, hy, hz}, sd[3] = {sdx, sdy, sdz}, st_t, sn[3];
                    int64_t ss = closest_hit(sc, so, sd, &st_t, sn, st);
                    l_shadow[tid] += 1;
                    int occluded = ss >= 0 && st_t > EPS && st_t < dist - EPS;
                    if (!occluded) {
                        double scat = sc->scattering[surf];
                        double diffuse = (1.0 / PI) * scat * facing;
                        double half[3];
                        normalize3(sdx - dir[0], sdy - dir[1], sdz - dir[2], half);
                        double cos_half = half[0] * n[0] + half[1] * n[1] + half[2] * n[2];
                        if (cos_half < 0.0) cos_half = 0.0;
                        double specular = ((p->specular_exponent + 2.0) / (8.0 * PI)) * (1.0 - scat) *
                                          pow(cos_half, p->specular_exponent);
                        double dmax = dist > p->irradiance_min_distance ? dist : p->irradiance_min_distance;
                        double inv = 1.0 / dmax;
                        double distance_term = (1.0 / (4.0 * PI)) * (inv * inv);
                        double source_cosine = -(fwd[0] * sdx + fwd[1] * sdy + fwd[2] * sdz);
                        double source_gain =
                            pow(fabs((1.0 - p->dipole_weight) + p->dipole_weight * source_cosine), p->dipole_power);
                        double rel_delay = (accum_distance + t + dist) / p->c - p->direct_delay;
                        double q = floor(rel_delay / p->bin_dur);
                        if (q >= 0.0 && q < (double)NBIN) {
                            int64_t bin = (int64_t)q;
                            double energy_sum = 0.0;
                            for (int bi = 0; bi < NB; ++bi) {
                                double e = ray_scale * source_gain * distance_term * (diffuse + specular) *
                                           sc->reflection[NB * surf + bi] * acc[bi];
                                echo[bi * NBIN + bin] += e;
                                if (ambi) {
                                    double *a = ambi + (size_t)bi * 4 * NBIN;
                                    a[0 * NBIN + bin] += e;
                                    a[1 * NBIN + bin] += e * p->directions[3 * ri];
                                    a[2 * NBIN + bin] += e * p->directions[3 * ri + 1];
                                    a[3 * NBIN + bin] += e * p->directions[3 * ri + 2];
                                }
                                energy_sum += e;
                            }
                            l_contrib[(size_t)tid * S + surf] += 1;
                            l_energy[(size_t)tid * S + surf] += energy_sum;
                        }
                    }
                }
            }
            for (int bi = 0; bi < NB; ++bi) acc[bi] *= sc->reflection[NB * surf + bi];
            accum_distance += t;
            origin[0] = hx; origin[1] = hy; origin[2] = hz;
            if (p->diffuse_random[bounce * R + ri] < sc->scattering[surf]) {
                int32_t idx = p->diffuse_indices[bounce * R + ri];
                double nd[3];
                diffuse_direction(p->diffuse_bank + 3 * idx, n[0], n[1], n[2], nd);
                dir[0] = nd[0]; dir[1] = nd[1]; dir[2] = nd[2];
            } else {
                double dot = dir[0] * n[0] + dir[1] * n[1] + dir[2] * n[2];
                double nd[3];
                normalize3(dir[0] - 2.0 * dot * n[0], dir[1] - 2.0 * dot * n[1], dir[2] - 2.0 * dot * n[2], nd);
                dir[0] = nd[0]; dir[1] = nd[1]; dir[2] = nd[2];
            }
            if (accum_distance > p->max_path_len) { alive = 0; break; }
        }
        if (alive) l_active[tid] += 1;
        if (out->ray_bounces) out->ray_bounces[ri] = queries;
    }

    memset(out->echogram, 0, sizeof(double) * NB * NBIN);
    if (amb) memset(out->ambisonic, 0, sizeof(double) * NB * 4 * NBIN);
    memset(out->hit_counts, 0, sizeof(int64_t) * S);
    memset(out->contrib_counts, 0, sizeof(int64_t) * S);
    memset(out->surface_energy, 0, sizeof(double) * S);
    out->actual_bounces = 0;
    out->active_count = 0;
    out->closest_queries = out->shadow_queries = out->nodes_visited = out->polygon_edges = 0;
    out->prims_tested[0] = out->prims_tested[1] = out->prims_tested[2] = 0;
    for (int ti = 0; ti < threads; ++ti) {
        out->active_count += l_active[ti];
        if (l_bounces[ti] > out->actual_bounces) out->actual_bounces = l_bounces[ti];
        for (int64_t si = 0; si < S; ++si) {
            out->hit_counts[si] += l_hits[(size_t)ti * S + si];
            out->contrib_counts[si] += l_contrib[(size_t)ti * S + si];
            out->surface_energy[si] += l_energy[(size_t)ti * S + si];
        }
        for (int64_t k = 0; k < NB * NBIN; ++k) out->echogram[k] += l_echo[(size_t)ti * NB * NBIN + k];
        if (amb)
            for (int64_t k = 0; k < NB * 4 * NBIN; ++k) out->ambisonic[k] += l_amb[(size_t)ti * NB * 4 * NBIN + k];
        out->closest_queries += l_closest[ti];
        out->shadow_queries += l_shadow[ti];
        out->nodes_visited += l_stats[ti].nodes;
        out->polygon_edges += l_stats[ti].edges;
        for (int k = 0; k < 3; ++k) out->prims_tested[k] += l_stats[ti].prims[k];
    }
    free(l_echo); free(l_amb); free(l_hits); free(l_contrib); free(l_energy); free(l_active);
    free(l_bounces); free(l_stats); free(l_closest); free(l_shadow);
    return 0;
}

/* steam_rt.py:4131-4146: one biquad section; state in double, output rounded to float32. */
static void biquad(const double *x, float *y, int64_t n, const double *co)
{
    double b0 = co[0], b1 = co[1], b2 = co[2], a1 = co[3], a2 = co[4];
    double x1 = 0.0, x2 = 0.0, y1 = 0.0, y2 = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double x0 = x[i];
        double y0 = b0 * x0 + b1 * x1 + b2 * x2 - a1 * y1 - a2 * y2;
        y[i] = (float)y0;
        x2 = x1; x1 = x0;
        y2 = y1; y1 = y0;
    }
}

/* Eight-pole low-pass: four cascaded sections, each fed the previous section's float32 output. */
static void lowpass8(const double *x, float *y, double *tmp, int64_t n, const double *sections)
{
    biquad(x, y, n, sections);
    for (int s = 1; s < 4; ++s) {
        for (int64_t i = 0; i < n; ++i) tmp[i] = (double)y[i];
        biquad(tmp, y, n, sections + 5 * s);
    }
}

/*
 * Echogram -> six band signals (steam_rt.py:2205-2232 and 3070-3083).
 * echogram_f32 != 0 means the echogram arrived as float32 (as the GPU
 * backends return it): numpy then evaluates sqrt(E / 4pi) and the 1e-9
 * threshold in float32.  air[6, bins] holds exp(-alpha * c * t_b) per bin,
 * computed by the caller with the reference's formula.  crossover[5][4][5]
 * are the low-pass section coefficients for the five crossover cutoffs.
 */
int oracle_synthesize(const double *echogram, int64_t echogram_f32, int64_t num_bins, int64_t samples_per_bin,
                      const double *air, const double *white, const double *crossover, float *out)
{
    const int64_t N = num_bins * samples_per_bin;
    double *raw = malloc(sizeof(double) * NB * N);
    double *tmp = malloc(sizeof(double) * N);
    float *lp_hi = malloc(sizeof(float) * N);
    float *lp_lo = malloc(sizeof(float) * N);
    double *amps = malloc(sizeof(double) * num_bins);
    if (!raw || !tmp || !lp_hi || !lp_lo || !amps) {
        free(raw); free(tmp); free(lp_hi); free(lp_lo); free(amps);
        return -2;
    }
    for (int bi = 0; bi < NB; ++bi) {
        for (int64_t b = 0; b < num_bins; ++b) {
            double e = echogram[bi * num_bins + b];
            if (echogram_f32) {
                float ef = (float)e;
                float cl = ef > 0.0f ? ef : 0.0f;
                float a = sqrtf(cl / (float)(4.0 * PI));
                amps[b] = ef < (float)1e-9 ? 0.0 : (double)a;
            } else {
                double cl = e > 0.0 ? e : 0.0;
                double a = sqrt(cl / (4.0 * PI));
                amps[b] = e < 1e-9 ? 0.0 : a;
            }
        }
        for (int64_t b = 0; b < num_bins; ++b) {
            double prev = b == 0 ? amps[b] : amps[b - 1];
            double g = air[bi * num_bins + b];
            for (int64_t k = 0; k < samples_per_bin; ++k) {
                double w = (double)k / (double)samples_per_bin;
                double seg = (1.0 - w) * prev + w * amps[b];
                seg = seg * g;
                int64_t i = b * samples_per_bin + k;
                raw[bi * N + i] = seg * white[i];
            }
        }
    }
    /* band 0: LP(c0); bands 1..4: LP(c_k) - LP(c_{k-1}); band 5: x - LP(c4) */
    lowpass8(raw, out, tmp, N, crossover);
    for (int bi = 1; bi < NB - 1; ++bi) {
        lowpass8(raw + bi * N, lp_hi, tmp, N, crossover + 20 * bi);
        lowpass8(raw + bi * N, lp_lo, tmp, N, crossover + 20 * (bi - 1));
        for (int64_t i = 0; i < N; ++i) out[bi * N + i] = lp_hi[i] - lp_lo[i];
    }
    lowpass8(raw + (NB - 1) * N, lp_lo, tmp, N, crossover + 20 * (NB - 2));
    for (int64_t i = 0; i < N; ++i) out[(NB - 1) * N + i] = (float)(raw[(NB - 1) * N + i] - (double)lp_lo[i]);
    free(raw); free(tmp); free(lp_hi); free(lp_lo); free(amps);
    return 0;
}

/* bandlimit_band_signals (steam_rt.py:3070-3083) on six float64 signals [6, n]. */
int oracle_bandlimit(const double *signals, int64_t n, const double *crossover, float *out)
{
    double *tmp = malloc(sizeof(double) * (n > 0 ? n : 1));
    float *lp_hi = malloc(sizeof(float) * (n > 0 ? n : 1));
    float *lp_lo = malloc(sizeof(float) * (n > 0 ? n : 1));
    if (!tmp || !lp_hi || !lp_lo) {
        free(tmp); free(lp_hi); free(lp_lo);
        return -2;
    }
    lowpass8(signals, out, tmp, n, crossover);
    for (int bi = 1; bi < NB - 1; ++bi) {
        lowpass8(signals + bi * n, lp_hi, tmp, n, crossover + 20 * bi);
        lowpass8(signals + bi * n, lp_lo, tmp, n, crossover + 20 * (bi - 1));
        for (int64_t i = 0; i < n; ++i) out[bi * n + i] = lp_hi[i] - lp_lo[i];
    }
    lowpass8(signals + (NB - 1) * n, lp_lo, tmp, n, crossover + 20 * (NB - 2));
    for (int64_t i = 0; i < n; ++i) out[(NB - 1) * n + i] = (float)(signals[(NB - 1) * n + i] - (double)lp_lo[i]);
    free(tmp); free(lp_hi); free(lp_lo);
    return 0;
}

/* One direct-form-I section y = b0*x + b1*x1 + b2*x2 - a1*y1 - a2*y2, left to right; state {x1, x2, y1, y2}. */
static double fdn_section(const double *co, double *st, double x)
{
    double y = co[0] * x + co[1] * st[0] + co[2] * st[1] - co[3] * st[2] - co[4] * st[3];
    st[1] = st[0];
    st[0] = x;
    st[3] = st[2];
    st[2] = y;
    return y;
}

/*
 * The sixteen-line feedback delay network of steam_rt.py:2235-2327, one
 * sample at a time in the reference's order: each line reads its delay
 * line and runs its absorptive sections (absorptive[line][band][5]); the
 * line outputs are mixed by an unnormalised Hadamard butterfly (strides 1,
 * 2, 4, ...) and written back scaled by 0.25 (plus the unit impulse at
 * sample 0); the output is the mean of the line outputs through the
 * Schroeder all-pass stages (gain 0.5) and the tone sections tone[band][5].
 */
int oracle_fdn_impulse(const int64_t *delays, int64_t num_delays, const double *absorptive, int64_t num_bands,
                       int64_t num_samples, const int64_t *allpass_delays, int64_t num_allpass, const double *tone,
                       double *out)
{
    int64_t max_delay = 0, max_allpass = 0;
    for (int64_t l = 0; l < num_delays; ++l) max_delay = delays[l] > max_delay ? delays[l] : max_delay;
    for (int64_t s = 0; s < num_allpass; ++s) max_allpass = allpass_delays[s] > max_allpass ? allpass_delays[s] : max_allpass;
    max_delay += 1;
    max_allpass += 1;
    double *lines = calloc((size_t)(num_delays * max_delay), sizeof(double));
    int64_t *pos = calloc((size_t)num_delays, sizeof(int64_t));
    double *delayed = calloc((size_t)num_delays, sizeof(double));
    double *mixed = calloc((size_t)num_delays, sizeof(double));
    double *line_state = calloc((size_t)(num_delays * num_bands * 4), sizeof(double));
    double *tone_state = calloc((size_t)(num_bands * 4), sizeof(double));
    double *ap = calloc((size_t)(num_allpass * max_allpass), sizeof(double));
    int64_t *ap_pos = calloc((size_t)(num_allpass > 0 ? num_allpass : 1), sizeof(int64_t));
    if (!lines || !pos || !delayed || !mixed || !line_state || !tone_state || !ap || !ap_pos) {
        free(lines); free(pos); free(delayed); free(mixed); free(line_state); free(tone_state); free(ap); free(ap_pos);
        return -2;
    }
    for (int64_t n = 0; n < num_samples; ++n) {
        for (int64_t l = 0; l < num_delays; ++l) {
            double v = lines[l * max_delay + pos[l]];
            for (int64_t b = 0; b < num_bands; ++b)
                v = fdn_section(absorptive + (l * num_bands + b) * 5, line_state + (l * num_bands + b) * 4, v);
            delayed[l] = v;
            mixed[l] = v;
        }
        for (int64_t stride = 1; stride < num_delays; stride *= 2) {
            for (int64_t base = 0; base < num_delays; base += 2 * stride) {
                for (int64_t o = 0; o < stride; ++o) {
                    double first = mixed[base + o], second = mixed[base + o + stride];
                    mixed[base + o] = first + second;
                    mixed[base + o + stride] = first - second;
                }
            }
        }
        double injection = n == 0 ? 1.0 : 0.0;
        for (int64_t l = 0; l < num_delays; ++l) {
            lines[l * max_delay + pos[l]] = injection + 0.25 * mixed[l];
            pos[l] += 1;
            if (pos[l] >= delays[l]) pos[l] = 0;
        }
        double value = 0.0;
        for (int64_t l = 0; l < num_delays; ++l) value += delayed[l];
        value /= (double)num_delays;
        for (int64_t s = 0; s < num_allpass; ++s) {
            double *buf = ap + s * max_allpass;
            double previous = buf[ap_pos[s]];
            double internal = value + 0.5 * previous;
            buf[ap_pos[s]] = internal;
            value = previous - 0.5 * internal;
            ap_pos[s] += 1;
            if (ap_pos[s] >= allpass_delays[s]) ap_pos[s] = 0;
        }
        for (int64_t b = 0; b < num_bands; ++b) value = fdn_section(tone + b * 5, tone_state + b * 4, value);
        out[n] = value;
    }
    free(lines); free(pos); free(delayed); free(mixed); free(line_state); free(tone_state); free(ap); free(ap_pos);
    return 0;
}
