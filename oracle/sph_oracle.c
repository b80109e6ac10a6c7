/*
 * sph_oracle.c -- CPU restatement of the reference's SPH hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this file's library, and only as the
 * checker / the timed CPU baseline.  The product (graphics_b200, libsphgpu)
 * never calls it.
 *
 * What it restates (reference = Artemisaturn/GRAPHICS, paths relative to its
 * Source/ directory):
 *   - uniform grid + linked-list neighbour search  SphBase.cpp:849-1089,
 *     SphBase.h:595-705 (cap NeigbStr::maxNeigbNum = 48, SphBase.h:630)
 *   - cubic spline kernel and gradient             SphBase.h:808-889
 *   - boundary (Akinci) volume                     SphBase.cpp:766-841
 *   - Euler-Cromer integration, outside removal    SphBase.cpp:377-402, 26-48
 *   - DFSPH: rho/alpha, non-pressure forces, constant-density and
 *     divergence-free Jacobi loops, step order     DFSPH.cpp:9-75, 84-1024,
 *                                                  1246-1475
 *   - WCSPH: Tait pressure and forces              WcSph.cpp:23-462
 *   - PCISPH predict/correct loop                  PciSph.cpp:98-505
 *   - IISPH multiphase (IISph_M)                   IISph_M.cpp:10-684
 *   - IISph, volume form (divergence-free and
 *     constant-volume loops, per-pair h)           IISph.cpp:14-545, 546-815,
 *                                                  1219-1570
 *
 * Arithmetic follows the reference expression by expression (evaluation order,
 * float/double promotions of std::pow), so that with `real` = float and no FMA
 * contraction (-ffp-contract=off) it reproduces the reference's float build.
 * Compiled twice: real=float (liboracle.so) and real=double (liboracle_f64.so).
 *
 * Deliberate differences from the reference, each switchable:
 *   - convergence sums are FP64 (the reference sums the DFSPH density error in
 *     float, DFSPH.cpp:227,627-631, which stalls at large N) unless
 *     OrcParams.float_err is set, which restores the reference's float sum;
 *   - every solver loop has an iteration cap (the DFSPH density loop has none
 *     in the reference, DFSPH.cpp:566);
 *   - the convergence goals are parameters (reference: 1e-4 relative for the
 *     density loop, DFSPH.cpp:225; 2.5 absolute for the divergence loop,
 *     DFSPH.cpp:762);
 *   - optional CFL time step dt = min(cfl*d/max|v|, dt_max) with an FP64 max
 *     (not in the reference).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_DOUBLE
typedef double real;
#define POWR(a, b) pow((a), (b))
#define SQRTR(a) sqrt(a)
#else
typedef float real;
#define POWR(a, b) powf((a), (b))
#define SQRTR(a) sqrtf(a)
#endif

#define ORC_CAP_MAX 256

typedef struct OrcParams {
    double spacing_r, smoothRadius_h, dt;
    double gravity[3];
    double densityErro_eta, soundSpeed_cs;
    double nu;
    double th_h, th_r, th_bt;
    double spaceMin[3], spaceMax[3];
    /* restatement controls (not reference parameters) */
    int cap;              /* neighbour cap, reference 48 */
    int float_err;        /* 1: reference float error sums */
    double df_density_goal; /* relative, reference 1e-4 */
    int df_density_min_iter, df_density_max_iter; /* reference 2, none */
    double df_div_goal_abs;  /* >0: absolute goal (reference 2.5) */
    double df_div_goal_rel;  /* used when abs <= 0: mean(div)*dt/rho0 */
    int df_div_min_iter, df_div_max_iter; /* reference 1, 30 (break at it>30) */
    int cfl;              /* 1: adaptive dt */
    double cfl_factor, dt_max, dt_min;
    double wc_gamma;      /* Tait exponent, reference 7 (WcSph.h:34) */
    double pci_eta; int pci_min_iter, pci_max_iter; /* PciSph.h:35 */
    double ii_omega, ii_eta_rel; int ii_min_iter, ii_max_iter;
    int ii_compat;        /* IISPH_M reference-compatibility bits (sph_oracle_pci_ii.inc) */
    /* IISph (volume form, sph_oracle_iisph.inc): FluidParticle /
     * BoundaryParticle::kinematicViscosity (SphBase.h:100,181, default 0.1)
     * and the loop bounds of IISph.cpp:550-555 (goal 1e-4, min 3, max 100)
     * and :1223-1227 (goal 1e-3, min 2, max 50) */
    double iv_kvisc, iv_kvisc_b, iv_cv_goal, iv_div_goal;
    int iv_cv_min_iter, iv_cv_max_iter, iv_div_min_iter, iv_div_max_iter;
} OrcParams;

typedef struct { int t, i; } PIdx; /* PartIdx, SphBase.h:596-617 */

typedef struct {
    int n;
    real d, rho0, visc_alpha, tension;
    real *pos, *vel, *vel_adv, *acce_adv, *acceleration, *DFalpha1, *n_surf;
    real *density, *DFalpha, *DFalpha2, *DFkappa, *DFkappaV, *density_adv, *divdev, *presure;
    /* PCISPH / IISPH */
    real *pos_pred, *acce_pressure, *dii, *sum_dijpj, *adv_vel, *acce_presure;
    real *aii, *rho_adv, *p_l, *p_l2;
    /* IISph (volume form): per-phase beta (SphBase.h:98; restDensity =
     * rho0 * beta) and per-particle state */
    real beta;
    real *adv_acc, *VF_alpha1;
    real *sphDensity, *VF_gamma, *VF_sphVolume, *VF_advVol, *VF_alpha, *VF_alpha2, *VF_kappa, *VF_kappaV,
        *VF_divdev;
    int *nnum; PIdx *nidx; real *ndis; /* neighbour lists, cap entries each */
    PIdx *next;
} OrcFluid;

typedef struct {
    int n, rigid;
    real d, visc_alpha, rho0;
    real *pos, *vel, *svel, *volume, *kerSumFromSelf, *force;
    /* dynamic rigid solid (SphSolid::dynamic, SphBase.h:330): body-frame
     * positions (innerPositions, SphBase.h:336) and the rigid state the
     * rigid-body world last reported: OpenGL column-major transform (float,
     * as btTransform::getOpenGLMatrix writes it), centre of mass, linear and
     * angular velocity (SphWithBullet.cpp:302-317) */
    int dynamic;
    real* inner;
    float T[16];
    real com[3], lin[3], ang[3];
    /* IISph (volume form) per-particle state */
    real *mass, *VF_gamma, *VF_sphVolume, *VF_advVol, *VF_alpha, *VF_alpha2, *VF_kappa, *VF_kappaV, *VF_divdev;
    int *nnum; PIdx *nidx; real *ndis;
    PIdx *next;
} OrcSolid;

typedef struct {
    OrcParams P;
    int nf, ns;
    OrcFluid F[8];
    OrcSolid S[16];
    /* grid, SphBase.h:682-705 */
    real gmin[3], divisor;
    int gnum[3], factor[3];
    int offset[27];
    long gcells;
    PIdx* gridFirst;
    real last_min[3], last_max[3], last_h;
    /* kernel constants, SphBase.h:789-791 */
    real ker_h, theta, thetah;
    long zeroDis, tooMany;
    int frame; double time;
    /* last-step statistics */
    int it_density, it_div, it_pci, it_ii;
    double err_density, err_div, err_pci, err_ii;
    real pci_delta, pci_last_dt, pci_last_sp, pci_last_h, pci_last_delta;
    int pci_init;
    int it_iv_div, it_iv_cv;
    double err_iv_div, err_iv_cv;
    /* the rigid-body world that stands in for Bullet (SphWithBullet::
     * updateSolids, SphWithBullet.cpp:180-224): per dynamic solid it receives
     * the joined force and torque and returns the new state, 25 doubles
     * (transform[16], com[3], linear[3], angular[3]); nonzero = failure */
    int (*rigid_fn)(void* user, int nsolids, const int* ids, const double* force, const double* torque,
                    double dt, double* states);
    void* rigid_user;
    int rigid_err;
} OrcScene;

/* ---------------- kernels, SphBase.h:808-889 ---------------- */
static void ker_update_numbers(OrcScene* s) {
    real h = (real)s->P.smoothRadius_h / 2;
    s->ker_h = h;
    s->theta = 1 / (real)M_PI / (h * h * h);
    s->thetah = 1 / (real)M_PI / (h * h * h) / h;
}
static inline real ker_W(const OrcScene* s, real r) {
    real q = r / s->ker_h, qm2 = 2 - q;
    return q <= 1 ? s->theta * (1 - (real)1.5 * q * q + (real)0.75 * q * q * q)
                  : s->theta * ((real)0.25 * qm2 * qm2 * qm2);
}
static inline real ker_W_grad(const OrcScene* s, real r) {
    real q = r / s->ker_h, qm2 = 2 - q;
    return q <= 1 ? s->thetah * (3 * q - (real)2.25 * q * q) : s->thetah * (real)0.75 * qm2 * qm2;
}
/* per-pair-h spline, SphBase.h:855-871 (boundary volumes use it) */
static inline real ker_W_h(real r, real h) {
    real q = r / h, qm2 = 2 - q;
    real th = 1 / (real)M_PI / (h * h * h);
    if (!(q >= 0 && q <= 2)) return 0;
    return q <= 1 ? th * (1 - (real)1.5 * q * q + (real)0.75 * q * q * q) : th * ((real)0.25 * qm2 * qm2 * qm2);
}

static inline real* fpos(OrcScene* s, PIdx p) {
    return p.t < 0 ? s->F[-p.t - 1].pos + 3 * (long)p.i : s->S[p.t - 1].pos + 3 * (long)p.i;
}
static inline real pd(OrcScene* s, PIdx p) { return p.t < 0 ? s->F[-p.t - 1].d : s->S[p.t - 1].d; }
static inline PIdx nextof(OrcScene* s, PIdx p) {
    return p.t < 0 ? s->F[-p.t - 1].next[p.i] : s->S[p.t - 1].next[p.i];
}
/* Vec23.h:170-171 */
static inline real dis_square(const real* a, const real* b) {
    return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
}

/* ---------------- grid, SphBase.cpp:963-1089 ---------------- */
static void grid_initialize(OrcScene* s) {
    real h = (real)s->P.smoothRadius_h;
    real smin[3], smax[3];
    for (int i = 0; i < 3; ++i) { smin[i] = (real)s->P.spaceMin[i]; smax[i] = (real)s->P.spaceMax[i]; }
    for (int i = 0; i < 3; ++i) s->gmin[i] = smin[i] - h * 2;
    s->divisor = 1 / h;
    for (int i = 0; i < 3; ++i) s->gnum[i] = (int)((smax[i] - smin[i] + h * 2) * s->divisor) + 2;
    for (int i = 0; i < 3; ++i) {
        s->factor[i] = 1;
        for (int j = 0; j < i; ++j) s->factor[i] *= s->gnum[j];
    }
    s->gcells = (long)s->gnum[0] * s->gnum[1] * s->gnum[2];
    free(s->gridFirst);
    s->gridFirst = (PIdx*)malloc(sizeof(PIdx) * s->gcells);
    int n = 0;
    for (int z = -1; z <= 1; ++z)
        for (int y = -1; y <= 1; ++y)
            for (int x = -1; x <= 1; ++x) s->offset[n++] = x * s->factor[0] + y * s->factor[1] + z * s->factor[2];
}

static inline long grid_of_pos(const OrcScene* s, const real* p) {
    int ix = (int)((p[0] - s->gmin[0]) * s->divisor);
    int iy = (int)((p[1] - s->gmin[1]) * s->divisor);
    int iz = (int)((p[2] - s->gmin[2]) * s->divisor);
    return (long)ix * s->factor[0] + (long)iy * s->factor[1] + (long)iz * s->factor[2];
}

static void grid_setup(OrcScene* s) {
    int same = 1;
    for (int i = 0; i < 3; ++i)
        if ((real)s->P.spaceMin[i] != s->last_min[i] || (real)s->P.spaceMax[i] != s->last_max[i]) same = 0;
    if ((real)s->P.smoothRadius_h != s->last_h) same = 0;
    if (!same || !s->gridFirst) {
        for (int i = 0; i < 3; ++i) { s->last_min[i] = (real)s->P.spaceMin[i]; s->last_max[i] = (real)s->P.spaceMax[i]; }
        s->last_h = (real)s->P.smoothRadius_h;
        grid_initialize(s);
    }
    for (long i = 0; i < s->gcells; ++i) { s->gridFirst[i].t = 0; s->gridFirst[i].i = -1; }
    /* solids first, then fluids; each particle pushed at the head of its cell
       list (SphBase.cpp:1033-1067) */
    for (int k = 0; k < s->ns; ++k) {
        OrcSolid* S = &s->S[k];
        for (int i = 0; i < S->n; ++i) {
            long g = grid_of_pos(s, S->pos + 3 * (long)i);
            S->next[i] = s->gridFirst[g];
            s->gridFirst[g].t = k + 1; s->gridFirst[g].i = i;
        }
    }
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        for (int i = 0; i < F->n; ++i) {
            long g = grid_of_pos(s, F->pos + 3 * (long)i);
            F->next[i] = s->gridFirst[g];
            s->gridFirst[g].t = -(k + 1); s->gridFirst[g].i = i;
        }
    }
}

/* SphBase.cpp:849-960 (neighbourSearch), RR_same for the rigid self test */
static void neighbour_search(OrcScene* s, int fluidPart, int solidPart, int RR_same) {
    grid_setup(s);
    const int cap = s->P.cap;
    long tooMany = 0;
    if (fluidPart)
        for (int k = 0; k < s->nf; ++k) {
            OrcFluid* F = &s->F[k];
            int t = -(k + 1);
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : tooMany)
            for (int ii = 0; ii < F->n; ++ii) {
                const real* pa = F->pos + 3 * (long)ii;
                int num = 0;
                PIdx* L = F->nidx + (long)ii * cap;
                real* D = F->ndis + (long)ii * cap;
                long jo = grid_of_pos(s, pa);
                for (int n = 0; n < 27; ++n)
                    for (PIdx j = s->gridFirst[jo + s->offset[n]]; j.t != 0; j = nextof(s, j)) {
                        if (j.t == t && j.i == ii) continue;
                        const real* pb = fpos(s, j);
                        real h = pd(s, j) + F->d;
                        real h2 = (real)pow(h, 2);
                        real len2 = dis_square(pa, pb);
                        if (len2 < h2) {
                            if (num < cap) { L[num] = j; D[num] = SQRTR(len2); ++num; }
                            else ++tooMany;
                        }
                    }
                F->nnum[ii] = num;
            }
        }
    if (solidPart)
        for (int k = 0; k < s->ns; ++k) {
            OrcSolid* S = &s->S[k];
            int t = k + 1;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : tooMany)
            for (int ii = 0; ii < S->n; ++ii) {
                const real* pa = S->pos + 3 * (long)ii;
                int num = 0;
                PIdx* L = S->nidx + (long)ii * cap;
                real* D = S->ndis + (long)ii * cap;
                long jo = grid_of_pos(s, pa);
                for (int n = 0; n < 27; ++n)
                    for (PIdx j = s->gridFirst[jo + s->offset[n]]; j.t != 0; j = nextof(s, j)) {
                        if (j.t == t && j.i == ii) continue;
                        if (!RR_same && S->rigid && j.t == t) continue;
                        const real* pb = fpos(s, j);
                        real h = pd(s, j) + S->d;
                        real h2 = (real)pow(h, 2);
                        real len2 = dis_square(pa, pb);
                        if (len2 < h2) {
                            if (num < cap) { L[num] = j; D[num] = SQRTR(len2); ++num; }
                            else ++tooMany;
                        }
                    }
                S->nnum[ii] = num;
            }
        }
    s->tooMany += tooMany;
}

/* SphBase.cpp:766-813 */
static void prepare_solid_part_weight(OrcScene* s) {
    neighbour_search(s, 0, 1, 1);
    const int cap = s->P.cap;
    for (int k = 0; k < s->ns; ++k) {
        OrcSolid* S = &s->S[k];
        for (int i = 0; i < S->n; ++i) {
            real h = S->d;
            real w0 = ker_W_h(0, h);
            const PIdx* L = S->nidx + (long)i * cap;
            const real* D = S->ndis + (long)i * cap;
            int n = S->nnum[i];
            if (S->rigid) {
                real sum = w0, sum2 = w0;
                for (int j = 0; j < n; ++j) {
                    if (L[j].t - 1 == k) { h = (S->d + pd(s, L[j])) / 2; sum += ker_W_h(D[j], h); }
                    if (L[j].t > 0) { h = (S->d + pd(s, L[j])) / 2; sum2 += ker_W_h(D[j], h); }
                }
                S->kerSumFromSelf[i] = sum;
                S->volume[i] = 1 / sum2;
            } else {
                real sum2 = w0;
                for (int j = 0; j < n; ++j)
                    if (L[j].t > 0) { h = (S->d + pd(s, L[j])) / 2; sum2 += ker_W_h(D[j], h); }
                S->kerSumFromSelf[i] = w0;
                S->volume[i] = 1 / sum2;
            }
        }
    }
}

/* SphBase.cpp:817-841 */
static void update_solid_part_weight(OrcScene* s) {
    const int cap = s->P.cap;
    for (int k = 0; k < s->ns; ++k) {
        OrcSolid* S = &s->S[k];
#pragma omp parallel for
        for (int i = 0; i < S->n; ++i) {
            const PIdx* L = S->nidx + (long)i * cap;
            const real* D = S->ndis + (long)i * cap;
            int n = S->nnum[i];
            real volume = S->kerSumFromSelf[i];
            for (int j = 0; j < n; ++j)
                if (L[j].t > 0) { real h = (S->d + pd(s, L[j])) / 2; volume += ker_W_h(D[j], h); }
            S->volume[i] = 1 / volume;
        }
    }
}

/* SphBase.h:193-194 inside(), Vec23.h:81-84 */
static inline int inside(const real* p, const real* mn, const real* mx) {
    return mn[0] <= p[0] && mn[1] <= p[1] && mn[2] <= p[2] && p[0] <= mx[0] && p[1] <= mx[1] && p[2] <= mx[2];
}

static void copy_fluid_particle(OrcFluid* F, int dst, int src) {
#define CP3(a) if (F->a) { F->a[3 * (long)dst] = F->a[3 * (long)src]; F->a[3 * (long)dst + 1] = F->a[3 * (long)src + 1]; F->a[3 * (long)dst + 2] = F->a[3 * (long)src + 2]; }
#define CP1(a) if (F->a) F->a[dst] = F->a[src];
    CP3(pos) CP3(vel) CP3(vel_adv) CP3(acce_adv) CP3(acceleration) CP3(DFalpha1) CP3(n_surf)
    CP3(pos_pred) CP3(acce_pressure) CP3(dii) CP3(sum_dijpj) CP3(adv_vel) CP3(acce_presure)
    CP1(density) CP1(DFalpha) CP1(DFalpha2) CP1(DFkappa) CP1(DFkappaV) CP1(density_adv) CP1(divdev)
    CP1(presure) CP1(aii) CP1(rho_adv) CP1(p_l) CP1(p_l2)
    CP3(adv_acc) CP3(VF_alpha1) CP1(sphDensity) CP1(VF_gamma) CP1(VF_sphVolume) CP1(VF_advVol) CP1(VF_alpha)
    CP1(VF_alpha2) CP1(VF_kappa) CP1(VF_kappaV) CP1(VF_divdev)
#undef CP3
#undef CP1
}

/* SphFluid::removeOutsideParts, SphBase.cpp:26-48 (swap compaction) */
static int remove_outside(OrcScene* s, OrcFluid* F) {
    if (!F->n) return 0;
    real mn[3], mx[3];
    for (int i = 0; i < 3; ++i) { mn[i] = (real)s->P.spaceMin[i]; mx[i] = (real)s->P.spaceMax[i]; }
    int num = F->n, f = 0, b = num - 1;
    while (f < b) {
        while (f < b && inside(F->pos + 3 * (long)f, mn, mx)) ++f;
        while (b > f && !inside(F->pos + 3 * (long)b, mn, mx)) --b;
        if (f < b) { copy_fluid_particle(F, f, b); ++f; --b; }
    }
    if (!inside(F->pos + 3 * (long)f, mn, mx)) --f;
    F->n = f + 1;
    return num - (f + 1);
}

/* Euler-Cromer, SphBase.cpp:377-402; use_acce_presure mirrors -DIISPH */
static void update_fluids(OrcScene* s, int use_acce_presure) {
    real dt = (real)s->P.dt;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        const real* a = use_acce_presure ? F->acce_presure : F->acceleration;
#pragma omp parallel for
        for (int i = 0; i < F->n; ++i) {
            real* v = F->vel + 3 * (long)i;
            real* x = F->pos + 3 * (long)i;
            if (use_acce_presure) {
                for (int c = 0; c < 3; ++c) v[c] = v[c] + a[3 * (long)i + c] * dt;
            } else {
                for (int c = 0; c < 3; ++c) v[c] += a[3 * (long)i + c] * dt;
            }
            for (int c = 0; c < 3; ++c) x[c] += v[c] * dt;
        }
        remove_outside(s, F);
    }
}

static inline real v0_of(const OrcScene* s) { return (real)pow((real)s->P.spacing_r, 3); }

/* ---------------- DFSPH ---------------- */

/* DF_constantDensitySolverFirst, DFSPH.cpp:84-193 */
static void df_first(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    for (int k = 0; k < s->ns; ++k) memset(s->S[k].force, 0, sizeof(real) * 3 * (size_t)s->S[k].n);
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0, wm0 = ker_W(s, 0) * fm0;
#pragma omp parallel for
        for (int i = 0; i < F->n; ++i) {
            const real* pa = F->pos + 3 * (long)i;
            real density = wm0, a1[3] = {0, 0, 0}, a2 = 0;
            const PIdx* L = F->nidx + (long)i * cap;
            const real* D = F->ndis + (long)i * cap;
            int n = F->nnum[i];
            for (int j = 0; j < n; ++j) {
                const real* pb = fpos(s, L[j]);
                real gs = -ker_W_grad(s, D[j]);
                real g[3];
                for (int c = 0; c < 3; ++c) g[c] = (pa[c] - pb[c]) * (gs / D[j]);
                if (L[j].t < 0) {
                    density += fm0 * ker_W(s, D[j]);
                    for (int c = 0; c < 3; ++c) a1[c] += g[c] * fm0;
                    a2 = (real)((double)a2 + pow(gs * fm0, 2));
                } else {
                    real vol = s->S[L[j].t - 1].volume[L[j].i];
                    density += rho0 * vol * ker_W(s, D[j]);
                    for (int c = 0; c < 3; ++c) a1[c] += g[c] * rho0 * vol;
                }
            }
            F->density[i] = density;
            F->DFalpha1[3 * (long)i] = a1[0]; F->DFalpha1[3 * (long)i + 1] = a1[1]; F->DFalpha1[3 * (long)i + 2] = a1[2];
            F->DFalpha2[i] = a2;
            real al = a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2] + a2;
            if (al < 1.0e-6) al = (real)1.0e-6;
            F->DFalpha[i] = density / al;
        }
    }
}

/* Boundary reaction of the viscosity term, `rb.force -= tmp` of
 * DF_fluidBoundExceptPressure (DFSPH.cpp:1334-1359), for fluid phase k.  The
 * reference adds it inside its OpenMP particle loop without synchronisation,
 * so with several threads its sums depend on the schedule; this serial pass
 * gives the one-thread order (particle, then neighbour) with the same
 * per-pair arithmetic as df_force_except_pressure. */
static void df_visc_reaction(OrcScene* s, int k) {
    const int cap = s->P.cap;
    OrcFluid* F = &s->F[k];
    real rho0 = F->rho0;
    real hs = (real)s->P.smoothRadius_h, nu = (real)s->P.nu;
    for (int i = 0; i < F->n; ++i) {
        const real* pa = F->pos + 3 * (long)i;
        const real* va = F->vel + 3 * (long)i;
        const PIdx* L = F->nidx + (long)i * cap;
        const real* D = F->ndis + (long)i * cap;
        int n = F->nnum[i];
        for (int j = 0; j < n; ++j) {
            if (L[j].t <= 0) continue;
            real dis = D[j];
            if (dis == 0) continue;
            OrcSolid* Sb = &s->S[L[j].t - 1];
            const real* pb = Sb->pos + 3 * (long)L[j].i;
            const real* sv = Sb->svel + 3 * (long)L[j].i;
            const real* bv = Sb->vel + 3 * (long)L[j].i;
            real* fb = Sb->force + 3 * (long)L[j].i;
            real xab[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
            real vol = Sb->volume[L[j].i];
            real s1 = -ker_W_grad(s, dis) / dis;
            real pro = (va[0] - sv[0] - bv[0]) * xab[0] + (va[1] - sv[1] - bv[1]) * xab[1] +
                       (va[2] - sv[2] - bv[2]) * xab[2];
            if (pro < 0) {
                real den = dis * dis + (real)0.01 * hs * hs;
                for (int c = 0; c < 3; ++c) {
                    real t = xab[c] * s1;
                    t = t * pro; t = t / den; t = t * (rho0 * vol); t = t / F->density[i]; t = t * 10; t = t * nu;
                    fb[c] = fb[c] - t;
                }
            }
        }
    }
}

/* Boundary reaction of one constant-density iteration, `p_b.force += acc_p`
 * (DFSPH.cpp:681-691), in the reference's one-thread order; acc_p is the
 * term the fluid particle's v_adv update subtracts (same arithmetic). */
static void df_pressure_reaction(OrcScene* s, OrcFluid* F) {
    const int cap = s->P.cap;
    real rho0 = F->rho0;
    for (int i = 0; i < F->n; ++i) {
        const real* pa = F->pos + 3 * (long)i;
        real ka = F->DFkappa[i] / F->density[i];
        const PIdx* L = F->nidx + (long)i * cap;
        const real* D = F->ndis + (long)i * cap;
        int n = F->nnum[i];
        for (int j = 0; j < n; ++j) {
            if (L[j].t <= 0) continue;
            OrcSolid* Sb = &s->S[L[j].t - 1];
            const real* pb = Sb->pos + 3 * (long)L[j].i;
            real* fb = Sb->force + 3 * (long)L[j].i;
            real vol = Sb->volume[L[j].i];
            real gs = -ker_W_grad(s, D[j]);
            for (int c = 0; c < 3; ++c) {
                real g = (pa[c] - pb[c]) * (gs / D[j]);
                real accp = g * rho0 * vol * ka;
                fb[c] += accp;
            }
        }
    }
}

/* DF_forceExceptPressure + ii_fluidPartForceExceptPressure_fsame/_fdiff and
 * DF_fluidBoundExceptPressure, DFSPH.cpp:1246-1359, 1419-1475 */
static void df_force_except_pressure(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    real hs = (real)s->P.smoothRadius_h, nu = (real)s->P.nu, cs = (real)s->P.soundSpeed_cs;
    real g[3] = {(real)s->P.gravity[0], (real)s->P.gravity[1], (real)s->P.gravity[2]};
    long zero = 0;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0, alpha = F->visc_alpha;
#pragma omp parallel for reduction(+ : zero)
        for (int i = 0; i < F->n; ++i) {
            const real* pa = F->pos + 3 * (long)i;
            const real* va = F->vel + 3 * (long)i;
            real* acc = F->acce_adv + 3 * (long)i;
            F->presure[i] = 0;
            acc[0] = g[0]; acc[1] = g[1]; acc[2] = g[2];
            const PIdx* L = F->nidx + (long)i * cap;
            const real* D = F->ndis + (long)i * cap;
            int n = F->nnum[i];
            for (int j = 0; j < n; ++j) {
                real dis = D[j];
                if (dis == 0) { ++zero; continue; }
                const real* pb = fpos(s, L[j]);
                real xab[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
                if (L[j].t < 0) {
                    OrcFluid* Fb = &s->F[-L[j].t - 1];
                    const real* vb = Fb->vel + 3 * (long)L[j].i;
                    real rhob = Fb->density[L[j].i];
                    real pro = (va[0] - vb[0]) * xab[0] + (va[1] - vb[1]) * xab[1] + (va[2] - vb[2]) * xab[2];
                    if (Fb == F) {
                        real s1 = -ker_W_grad(s, dis) / dis;
                        if (pro < 0) {
                            real den = dis * dis + (real)0.01 * hs * hs;
                            for (int c = 0; c < 3; ++c) {
                                real t = xab[c] * s1;
                                t = t * pro; t = t / den; t = t * fm0; t = t / rhob; t = t * 10; t = t * nu;
                                acc[c] += t;
                            }
                        }
                    } else {
                        real fmb = v0 * Fb->rho0, al = (alpha + Fb->visc_alpha) / 2;
                        real grad = -ker_W_grad(s, dis) / dis, acce = 0;
                        if (pro < 0) {
                            real nu2 = 2 * al * hs * cs / (F->density[i] + rhob);
                            real pi = -nu2 * pro / (dis * dis + (real)0.01 * hs * hs);
                            acce += grad * (-(fm0 + fmb) / 2 * pi);
                        }
                        if (acce) for (int c = 0; c < 3; ++c) acc[c] += xab[c] * acce;
                    }
                } else {
                    OrcSolid* Sb = &s->S[L[j].t - 1];
                    const real* sv = Sb->svel + 3 * (long)L[j].i;
                    const real* bv = Sb->vel + 3 * (long)L[j].i;
                    real vol = Sb->volume[L[j].i];
                    real s1 = -ker_W_grad(s, dis) / dis;
                    real pro = (va[0] - sv[0] - bv[0]) * xab[0] + (va[1] - sv[1] - bv[1]) * xab[1] +
                               (va[2] - sv[2] - bv[2]) * xab[2];
                    if (pro < 0) {
                        real den = dis * dis + (real)0.01 * hs * hs;
                        for (int c = 0; c < 3; ++c) {
                            real t = xab[c] * s1;
                            t = t * pro; t = t / den; t = t * (rho0 * vol); t = t / F->density[i]; t = t * 10; t = t * nu;
                            acc[c] += t;
                        }
                    }
                }
            }
        }
        df_visc_reaction(s, k);
    }
    s->zeroDis += zero;
}

/* DF_constantDensitySolverSecond, DFSPH.cpp:195-738 (vorticity options off) */
static void df_second(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    real dt = (real)s->P.dt;
    df_force_except_pressure(s);
    s->it_density = 0; s->err_density = 0;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0;
        int num = F->n;
        double goal = s->P.df_density_goal;
        double errorRate = 1;
        int it = 0;
#pragma omp parallel for
        for (int i = 0; i < num; ++i)
            for (int c = 0; c < 3; ++c) F->vel_adv[3 * (long)i + c] = F->vel[3 * (long)i + c] + F->acce_adv[3 * (long)i + c] * dt;
        while (((s->P.float_err ? ((real)errorRate > (real)goal) : (errorRate > goal)) ||
                it < s->P.df_density_min_iter) && it < s->P.df_density_max_iter) {
            /* 2.1 density_adv */
#pragma omp parallel for
            for (int i = 0; i < num; ++i) {
                const real* pa = F->pos + 3 * (long)i;
                const real* va = F->vel_adv + 3 * (long)i;
                real dadv = F->density[i];
                const PIdx* L = F->nidx + (long)i * cap;
                const real* D = F->ndis + (long)i * cap;
                int n = F->nnum[i];
                for (int j = 0; j < n; ++j) {
                    const real* pb = fpos(s, L[j]);
                    real gs = -ker_W_grad(s, D[j]);
                    real g[3] = {(pa[0] - pb[0]) * (gs / D[j]), (pa[1] - pb[1]) * (gs / D[j]), (pa[2] - pb[2]) * (gs / D[j])};
                    if (L[j].t < 0) {
                        const real* vb = s->F[-L[j].t - 1].vel_adv + 3 * (long)L[j].i;
                        real dot = g[0] * (va[0] - vb[0]) + g[1] * (va[1] - vb[1]) + g[2] * (va[2] - vb[2]);
                        dadv += dot * fm0 * dt;
                    } else {
                        OrcSolid* Sb = &s->S[L[j].t - 1];
                        const real* vb = Sb->svel + 3 * (long)L[j].i;
                        real dot = g[0] * (va[0] - vb[0]) + g[1] * (va[1] - vb[1]) + g[2] * (va[2] - vb[2]);
                        dadv += dot * rho0 * Sb->volume[L[j].i] * dt;
                    }
                }
                if (dadv < rho0) dadv = rho0;
                F->density_adv[i] = dadv;
            }
            double sum;
            if (s->P.float_err) {
                real fs = 0;
                for (int i = 0; i < num; ++i) fs += F->density_adv[i];
                sum = fs;
            } else {
                sum = 0;
#pragma omp parallel for reduction(+ : sum)
                for (int i = 0; i < num; ++i) sum += (double)F->density_adv[i];
            }
            /* 2.2 kappa */
#pragma omp parallel for
            for (int i = 0; i < num; ++i)
                F->DFkappa[i] = (real)((double)(F->density_adv[i] - rho0) / pow(dt, 2) * F->DFalpha[i]);
            /* 2.3 vel_adv */
#pragma omp parallel for
            for (int i = 0; i < num; ++i) {
                const real* pa = F->pos + 3 * (long)i;
                real* va = F->vel_adv + 3 * (long)i;
                real ka = F->DFkappa[i] / F->density[i];
                const PIdx* L = F->nidx + (long)i * cap;
                const real* D = F->ndis + (long)i * cap;
                int n = F->nnum[i];
                for (int j = 0; j < n; ++j) {
                    const real* pb = fpos(s, L[j]);
                    real gs = -ker_W_grad(s, D[j]);
                    real g[3] = {(pa[0] - pb[0]) * (gs / D[j]), (pa[1] - pb[1]) * (gs / D[j]), (pa[2] - pb[2]) * (gs / D[j])};
                    if (L[j].t < 0) {
                        OrcFluid* Fb = &s->F[-L[j].t - 1];
                        real kk = ka + Fb->DFkappa[L[j].i] / Fb->density[L[j].i];
                        for (int c = 0; c < 3; ++c) va[c] = va[c] - (g[c] * fm0 * kk * dt);
                    } else {
                        OrcSolid* Sb = &s->S[L[j].t - 1];
                        real vol = Sb->volume[L[j].i];
                        for (int c = 0; c < 3; ++c) {
                            real accp = g[c] * rho0 * vol * ka;
                            va[c] = va[c] - (accp * dt);
                        }
                    }
                }
            }
            df_pressure_reaction(s, F);
            if (s->P.float_err) {
                real fs = (real)sum;
                errorRate = ((fs / num) - rho0) / rho0;
            } else {
                errorRate = ((sum / num) - rho0) / rho0;
            }
            ++it;
        }
        /* 2.4 integrate */
#pragma omp parallel for
        for (int i = 0; i < num; ++i)
            for (int c = 0; c < 3; ++c) {
                F->vel[3 * (long)i + c] = F->vel_adv[3 * (long)i + c];
                F->pos[3 * (long)i + c] += F->vel[3 * (long)i + c] * dt;
            }
        remove_outside(s, F);
        if (it > s->it_density) s->it_density = it;
        if (errorRate > s->err_density || k == 0) s->err_density = errorRate;
    }
    /* acceleration-per-density sums -> forces, with the mass of phase 0
     * (DFSPH.cpp:723-737) */
    if (s->nf > 0) {
        real fm0 = v0 * s->F[0].rho0;
        for (int k = 0; k < s->ns; ++k) {
            OrcSolid* S = &s->S[k];
            for (long i = 0; i < 3L * S->n; ++i) S->force[i] = S->force[i] * fm0;
        }
    }
}

/* DF_divergenceFreeSolver, DFSPH.cpp:740-1024 (vorticity options off) */
static void df_divergence_free(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    real dt = (real)s->P.dt;
    s->it_div = 0; s->err_div = 0;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0;
        int num = F->n, it = 0;
        double aver = 0, goal_abs = s->P.df_div_goal_abs;
        double crit = 0;
        for (;;) {
            /* reference: while (aver > goal || it < min) { if (it > max) break; ... }
               with max = 30 (DFSPH.cpp:764-773) */
            if (!(crit > 0 || it < s->P.df_div_min_iter)) break;
            if (it > s->P.df_div_max_iter) break;
#pragma omp parallel for
            for (int i = 0; i < num; ++i) {
                const real* pa = F->pos + 3 * (long)i;
                const real* va = F->vel_adv + 3 * (long)i;
                real dd = 0;
                const PIdx* L = F->nidx + (long)i * cap;
                const real* D = F->ndis + (long)i * cap;
                int n = F->nnum[i];
                for (int j = 0; j < n; ++j) {
                    const real* pb = fpos(s, L[j]);
                    real gs = -ker_W_grad(s, D[j]);
                    real g[3] = {(pa[0] - pb[0]) * (gs / D[j]), (pa[1] - pb[1]) * (gs / D[j]), (pa[2] - pb[2]) * (gs / D[j])};
                    if (L[j].t < 0) {
                        const real* vb = s->F[-L[j].t - 1].vel_adv + 3 * (long)L[j].i;
                        real dot = g[0] * (va[0] - vb[0]) + g[1] * (va[1] - vb[1]) + g[2] * (va[2] - vb[2]);
                        dd += dot * fm0;
                    } else {
                        OrcSolid* Sb = &s->S[L[j].t - 1];
                        const real* vb = Sb->svel + 3 * (long)L[j].i;
                        real dot = g[0] * (va[0] - vb[0]) + g[1] * (va[1] - vb[1]) + g[2] * (va[2] - vb[2]);
                        dd += dot * (rho0 * Sb->volume[L[j].i]);
                    }
                }
                if (dd < 0 || (F->density[i] + dd * dt) < rho0) dd = 0;
                F->divdev[i] = dd;
                F->DFkappaV[i] = dd * F->DFalpha[i] / dt;
            }
#pragma omp parallel for
            for (int i = 0; i < num; ++i) {
                const real* pa = F->pos + 3 * (long)i;
                real* va = F->vel_adv + 3 * (long)i;
                real ka = F->DFkappaV[i] / F->density[i];
                const PIdx* L = F->nidx + (long)i * cap;
                const real* D = F->ndis + (long)i * cap;
                int n = F->nnum[i];
                for (int j = 0; j < n; ++j) {
                    const real* pb = fpos(s, L[j]);
                    real gs = -ker_W_grad(s, D[j]);
                    real g[3] = {(pa[0] - pb[0]) * (gs / D[j]), (pa[1] - pb[1]) * (gs / D[j]), (pa[2] - pb[2]) * (gs / D[j])};
                    if (L[j].t < 0) {
                        OrcFluid* Fb = &s->F[-L[j].t - 1];
                        real kk = ka + Fb->DFkappaV[L[j].i] / Fb->density[L[j].i];
                        for (int c = 0; c < 3; ++c) va[c] = va[c] - (g[c] * fm0 * kk * dt);
                    } else {
                        real vol = s->S[L[j].t - 1].volume[L[j].i];
                        for (int c = 0; c < 3; ++c) va[c] = va[c] - (g[c] * rho0 * vol * ka * dt);
                    }
                }
            }
            if (s->P.float_err) {
                real fa = 0;
                for (int i = 0; i < num; ++i) fa += F->divdev[i];
                fa = fa / num;
                aver = fa;
            } else {
                double sum = 0;
#pragma omp parallel for reduction(+ : sum)
                for (int i = 0; i < num; ++i) sum += (double)F->divdev[i];
                aver = sum / num;
            }
            if (s->P.float_err && goal_abs > 0)
                crit = (real)aver > (real)goal_abs;
            else
                crit = goal_abs > 0 ? (aver > goal_abs ? 1 : 0) : (aver * dt / rho0 > s->P.df_div_goal_rel ? 1 : 0);
            ++it;
        }
#pragma omp parallel for
        for (int i = 0; i < num; ++i)
            for (int c = 0; c < 3; ++c) F->vel[3 * (long)i + c] = F->vel_adv[3 * (long)i + c];
        if (it > s->it_div) s->it_div = it;
        double e = goal_abs > 0 ? aver : aver * dt / rho0;
        if (e > s->err_div || k == 0) s->err_div = e;
    }
}

/* CFL time step (new; the reference has a fixed dt): dt = cfl * d / max|v|
 * with the maximum taken in FP64, clamped to [dt_min, dt_max]. */
static void cfl_dt(OrcScene* s) {
    double vmax = 0;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        for (int i = 0; i < F->n; ++i) {
            double a = F->vel[3 * (long)i], b = F->vel[3 * (long)i + 1], c = F->vel[3 * (long)i + 2];
            double m = sqrt(a * a + b * b + c * c);
            if (m > vmax) vmax = m;
        }
    }
    double d = s->nf ? (double)s->F[0].d : s->P.spacing_r;
    double dt = vmax > 0 ? s->P.cfl_factor * d / vmax : s->P.dt_max;
    if (dt > s->P.dt_max) dt = s->P.dt_max;
    if (dt < s->P.dt_min) dt = s->P.dt_min;
    s->P.dt = (double)(float)dt;
}

/* SphSolid::updatePaticles(centerOfMass, tranform, linearVelocity,
 * angularVelocity), SphBase.cpp:95-128 (3-D branch): position = transform *
 * innerPosition with the homogeneous divide, velocity = v + w x (x - com). */
static void solid_update_particles(OrcSolid* S) {
    const float* t = S->T;
    for (int i = 0; i < S->n; ++i) {
        const real* p0 = S->inner + 3 * (long)i;
        real* bp = S->pos + 3 * (long)i;
        real* bv = S->vel + 3 * (long)i;
        bp[0] = t[0] * p0[0] + t[4] * p0[1] + t[8] * p0[2] + t[12];
        bp[1] = t[1] * p0[0] + t[5] * p0[1] + t[9] * p0[2] + t[13];
        bp[2] = t[2] * p0[0] + t[6] * p0[1] + t[10] * p0[2] + t[14];
        real alpha = t[3] * p0[0] + t[7] * p0[1] + t[11] * p0[2] + t[15];
        bp[0] /= alpha; bp[1] /= alpha; bp[2] /= alpha;
        real r[3] = {bp[0] - S->com[0], bp[1] - S->com[1], bp[2] - S->com[2]};
        /* vec3::cross, Vec23.h:142-143 */
        real w[3] = {S->ang[1] * r[2] - S->ang[2] * r[1], S->ang[2] * r[0] - S->ang[0] * r[2],
                     S->ang[0] * r[1] - S->ang[1] * r[0]};
        bv[0] = S->lin[0] + w[0]; bv[1] = S->lin[1] + w[1]; bv[2] = S->lin[2] + w[2];
    }
}

/* SphSolid::rigidForceJoin, SphBase.cpp:131-143: total force and the torque
 * about the centre of mass, summed in particle order. */
static void rigid_force_join(const OrcSolid* S, const real* com, real* tf, real* tt) {
    tf[0] = tf[1] = tf[2] = 0; tt[0] = tt[1] = tt[2] = 0;
    for (int i = 0; i < S->n; ++i) {
        const real* f = S->force + 3 * (long)i;
        const real* x = S->pos + 3 * (long)i;
        real r[3] = {x[0] - com[0], x[1] - com[1], x[2] - com[2]};
        tf[0] += f[0]; tf[1] += f[1]; tf[2] += f[2];
        tt[0] += r[1] * f[2] - r[2] * f[1];
        tt[1] += r[2] * f[0] - r[0] * f[2];
        tt[2] += r[0] * f[1] - r[1] * f[0];
    }
}

static void solid_set_state(OrcSolid* S, const double* st) {
    for (int c = 0; c < 16; ++c) S->T[c] = (float)st[c];
    for (int c = 0; c < 3; ++c) {
        S->com[c] = (real)(float)st[16 + c];
        S->lin[c] = (real)(float)st[19 + c];
        S->ang[c] = (real)(float)st[22 + c];
    }
}

/* SphWithBullet::updateSolids, SphWithBullet.cpp:180-224, with the rigid-body
 * world behind s->rigid_fn: join each dynamic solid's force and torque about
 * its current centre of mass, let the world advance the bodies by dt, then
 * move the boundary particles with the returned states.  Without a world the
 * bodies keep their states. */
static void update_solids(OrcScene* s) {
    int ids[16], nd = 0;
    double force[48], torque[48], states[16 * 25];
    for (int k = 0; k < s->ns; ++k) {
        OrcSolid* S = &s->S[k];
        if (!S->dynamic) continue;
        real tf[3], tt[3];
        rigid_force_join(S, S->com, tf, tt);
        for (int c = 0; c < 3; ++c) { force[3 * nd + c] = tf[c]; torque[3 * nd + c] = tt[c]; }
        for (int c = 0; c < 16; ++c) states[25 * nd + c] = S->T[c];
        for (int c = 0; c < 3; ++c) {
            states[25 * nd + 16 + c] = S->com[c];
            states[25 * nd + 19 + c] = S->lin[c];
            states[25 * nd + 22 + c] = S->ang[c];
        }
        ids[nd++] = k;
    }
    if (!nd) return;
    if (s->rigid_fn && s->rigid_fn(s->rigid_user, nd, ids, force, torque, (double)(real)s->P.dt, states))
        s->rigid_err = 1;
    for (int j = 0; j < nd; ++j) {
        OrcSolid* S = &s->S[ids[j]];
        solid_set_state(S, states + 25 * j);
        solid_update_particles(S);
    }
}

/* DFSPH::sphStep, DFSPH.cpp:45-62, followed by runOneStep's bookkeeping
 * (SphBase.cpp:348-354) */
static void df_step(OrcScene* s) {
    if (s->frame == 0) {
        neighbour_search(s, 1, 1, 0);
        update_solid_part_weight(s);
        df_first(s);
    }
    if (s->P.cfl) cfl_dt(s);
    df_second(s);
    update_solids(s);
    neighbour_search(s, 1, 1, 0);
    update_solid_part_weight(s);
    df_first(s);
    df_divergence_free(s);
    s->frame += 1;
    s->time += (real)s->P.dt;
}

/* ---------------- WCSPH ---------------- */

/* WcSph::wc_computePressure, WcSph.cpp:99-153 */
static void wc_pressure(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    real gamma = (real)s->P.wc_gamma, cs = (real)s->P.soundSpeed_cs, thh = (real)s->P.th_h;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0, wm0 = ker_W(s, 0) * fm0;
        real B = rho0 * cs * cs / gamma;
#pragma omp parallel for
        for (int i = 0; i < F->n; ++i) {
            real density = wm0;
            const PIdx* L = F->nidx + (long)i * cap;
            const real* D = F->ndis + (long)i * cap;
            int n = F->nnum[i];
            for (int j = 0; j < n; ++j) {
                if (L[j].t < 0) density += fm0 * ker_W(s, D[j]);
                else density += rho0 * s->S[L[j].t - 1].volume[L[j].i] * ker_W(s, D[j]);
            }
            F->density[i] = density;
            real p = B * (POWR(density / rho0, gamma) - 1);
            if (p < 0) p = 0;
            F->presure[i] = p;
        }
    }
    /* The surface normal n_i = h sum_j m/rho_j gradW_ij (WcSph.cpp:124-137)
     * with this step's densities: the reference reads the neighbours'
     * densities in the loop that writes them, so its value depends on the
     * thread schedule (it vanishes for m_TH.h = 0, the plain method). */
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real fm0 = F->rho0 * v0;
#pragma omp parallel for
        for (int i = 0; i < F->n; ++i) {
            const real* pa = F->pos + 3 * (long)i;
            real ni[3] = {0, 0, 0};
            const PIdx* L = F->nidx + (long)i * cap;
            const real* D = F->ndis + (long)i * cap;
            int n = F->nnum[i];
            for (int j = 0; j < n; ++j) {
                if (L[j].t >= 0) continue;
                const real* pb = fpos(s, L[j]);
                real gs = -ker_W_grad(s, D[j]) / D[j];
                real rb = s->F[-L[j].t - 1].density[L[j].i];
                for (int c = 0; c < 3; ++c) ni[c] += (pa[c] - pb[c]) * gs * (fm0 / rb);
            }
            for (int c = 0; c < 3; ++c) F->n_surf[3 * (long)i + c] = ni[c] * thh;
        }
    }
}

/* WcSph::wc_computeForce with wc_fluidPartForce_fsame/_fdiff/_bound,
 * WcSph.cpp:156-312, 364-436 (surface tension and adhesion included; they
 * vanish when m_TH.r = m_TH.bt = m_TH.h = 0) */
static void wc_force(OrcScene* s) {
    const int cap = s->P.cap;
    real v0 = v0_of(s);
    real hs = (real)s->P.smoothRadius_h, cs = (real)s->P.soundSpeed_cs;
    real thh = (real)s->P.th_h, thr = (real)s->P.th_r, thbt = (real)s->P.th_bt;
    real g[3] = {(real)s->P.gravity[0], (real)s->P.gravity[1], (real)s->P.gravity[2]};
    long zero = 0;
    for (int k = 0; k < s->nf; ++k) {
        OrcFluid* F = &s->F[k];
        real rho0 = F->rho0, fm0 = rho0 * v0, alpha = F->visc_alpha;
#pragma omp parallel for reduction(+ : zero)
        for (int i = 0; i < F->n; ++i) {
            const real* pa = F->pos + 3 * (long)i;
            const real* va = F->vel + 3 * (long)i;
            real* acc = F->acceleration + 3 * (long)i;
            real ra = F->density[i], pra = F->presure[i];
            acc[0] = g[0]; acc[1] = g[1]; acc[2] = g[2];
            const PIdx* L = F->nidx + (long)i * cap;
            const real* D = F->ndis + (long)i * cap;
            int n = F->nnum[i];
            for (int j = 0; j < n; ++j) {
                real dis = D[j];
                if (dis == 0) { ++zero; continue; }
                const real* pb = fpos(s, L[j]);
                real xab[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
                real grad = -ker_W_grad(s, dis) / dis;
                if (L[j].t < 0) {
                    OrcFluid* Fb = &s->F[-L[j].t - 1];
                    const real* vb = Fb->vel + 3 * (long)L[j].i;
                    real rb = Fb->density[L[j].i], prb = Fb->presure[L[j].i];
                    real pro = (va[0] - vb[0]) * xab[0] + (va[1] - vb[1]) * xab[1] + (va[2] - vb[2]) * xab[2];
                    if (Fb == F) {
                        real acce = grad * (-fm0 * (pra / (ra * ra) + prb / (rb * rb)));
                        if (pro < 0) {
                            real nu = 2 * alpha * hs * cs / (ra + rb);
                            real pi = -nu * pro / (dis * dis + (real)0.01 * hs * hs);
                            acce += grad * (-fm0 * pi);
                        }
                        for (int c = 0; c < 3; ++c) acc[c] += xab[c] * acce;
                        /* cohesion + curvature, WcSph.cpp:188-210 */
                        real Kij = 2 * 1000.0f / (ra + rb);
                        real C = 0;
                        if (2 * dis > thh && dis <= thh)
                            C = (32.0f / (3.14f * powf(thh, 9.0f))) * powf(thh - dis, 3.0f) * powf(dis, 3.0f);
                        else if (dis > 0 && 2 * dis <= thh)
                            C = (32.0f / (3.14f * powf(thh, 9.0f))) *
                                (2 * powf(thh - dis, 3.0f) * powf(dis, 3.0f) - powf(thh, 6.0f) / 64.0f);
                        real acce_coh = -thr * fm0 * C / dis;
                        real acce_cur = -thr;
                        const real* na = F->n_surf + 3 * (long)i;
                        const real* nb = Fb->n_surf + 3 * (long)L[j].i;
                        for (int c = 0; c < 3; ++c) {
                            real st = (xab[c] * acce_coh + (na[c] - nb[c]) * acce_cur) * Kij;
                            acc[c] += st;
                        }
                    } else {
                        real fmb = v0 * Fb->rho0, al = (alpha + Fb->visc_alpha) / 2;
                        real da = ra / fm0, db = rb / fmb;
                        real acce = grad * (-1 / fm0 * (pra / (da * da) + prb / (db * db)));
                        if (pro < 0) {
                            real nu = 2 * al * hs * cs / (ra + rb);
                            real pi = -nu * pro / (dis * dis + (real)0.01 * hs * hs);
                            acce += grad * (-(fm0 + fmb) / 2 * pi);
                        }
                        for (int c = 0; c < 3; ++c) acc[c] += xab[c] * acce;
                    }
                } else {
                    OrcSolid* Sb = &s->S[L[j].t - 1];
                    real vol = Sb->volume[L[j].i];
                    const real* vb = Sb->vel + 3 * (long)L[j].i;
                    real acce = 0;
                    if (pra > 0) acce += grad * (-rho0 * vol * (pra / (ra * ra) * 2));
                    real pro = (va[0] - vb[0]) * xab[0] + (va[1] - vb[1]) * xab[1] + (va[2] - vb[2]) * xab[2];
                    if (pro < 0) {
                        real nu = 2 * Sb->visc_alpha * hs * cs / (ra * 2);
                        real pi = -nu * pro / (dis * dis + (real)0.01 * hs * hs);
                        acce += grad * (-rho0 * vol * pi);
                    }
                    for (int c = 0; c < 3; ++c) acc[c] += xab[c] * acce;
                    /* adhesion, WcSph.cpp:300-311 */
                    real A = 0;
                    if (2 * dis > thh && dis <= thh)
                        A = 0.007f / (powf(thh, 3.25f)) * powf((-4 * dis * dis / thh + 6 * dis - 2 * thh), 0.25f);
                    real acce_adh = -thbt * rho0 * vol * A / dis;
                    for (int c = 0; c < 3; ++c) acc[c] += xab[c] * acce_adh;
                }
            }
        }
    }
    s->zeroDis += zero;
}

/* WcSph::sphStep, WcSph.cpp:23-96 */
static void wc_step(OrcScene* s) {
    neighbour_search(s, 1, 1, 0);
    update_solid_part_weight(s);
    wc_pressure(s);
    wc_force(s);
    update_fluids(s, 0);
    s->frame += 1;
    s->time += (real)s->P.dt;
}

#include "sph_oracle_pci_ii.inc"
#include "sph_oracle_iisph.inc"

/* ---------------- C interface ---------------- */

#define ALLOC3(p, n) p = (real*)calloc(3 * (size_t)(n) + 3, sizeof(real))
#define ALLOC1(p, n) p = (real*)calloc((size_t)(n) + 1, sizeof(real))

void* orc_create(const OrcParams* p) {
    OrcScene* s = (OrcScene*)calloc(1, sizeof(OrcScene));
    s->P = *p;
    if (s->P.cap <= 0 || s->P.cap > ORC_CAP_MAX) s->P.cap = 48;
    s->last_min[0] = 1; s->last_max[0] = -1; s->last_h = -1;
    ker_update_numbers(s);
    return s;
}

void orc_set_params(void* h, const OrcParams* p) {
    OrcScene* s = (OrcScene*)h;
    int cap = s->P.cap;
    s->P = *p;
    s->P.cap = cap; /* the cap sizes the neighbour arrays; fixed at creation */
    ker_update_numbers(s);
}

static void free_fluid(OrcFluid* F) {
    real* arrs[] = {F->pos, F->vel, F->vel_adv, F->acce_adv, F->acceleration, F->DFalpha1, F->n_surf,
                    F->density, F->DFalpha, F->DFalpha2, F->DFkappa, F->DFkappaV, F->density_adv, F->divdev,
                    F->presure, F->pos_pred, F->acce_pressure, F->dii, F->sum_dijpj, F->adv_vel,
                    F->acce_presure, F->aii, F->rho_adv, F->p_l, F->p_l2, F->ndis,
                    F->adv_acc, F->VF_alpha1, F->sphDensity, F->VF_gamma, F->VF_sphVolume, F->VF_advVol,
                    F->VF_alpha, F->VF_alpha2, F->VF_kappa, F->VF_kappaV, F->VF_divdev};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
    free(F->nnum); free(F->nidx); free(F->next);
}

void orc_destroy(void* h) {
    OrcScene* s = (OrcScene*)h;
    for (int k = 0; k < s->nf; ++k) free_fluid(&s->F[k]);
    for (int k = 0; k < s->ns; ++k) {
        OrcSolid* S = &s->S[k];
        free(S->pos); free(S->vel); free(S->svel); free(S->volume); free(S->kerSumFromSelf); free(S->force);
        free(S->inner);
        free(S->mass); free(S->VF_gamma); free(S->VF_sphVolume); free(S->VF_advVol); free(S->VF_alpha);
        free(S->VF_alpha2); free(S->VF_kappa); free(S->VF_kappaV); free(S->VF_divdev);
        free(S->nnum); free(S->nidx); free(S->ndis); free(S->next);
    }
    free(s->gridFirst);
    free(s);
}

int orc_add_solid(void* h, int n, const double* xyz, double d, double visc_alpha, double rho0, int prepare) {
    OrcScene* s = (OrcScene*)h;
    if (s->ns >= 16) return -1;
    OrcSolid* S = &s->S[s->ns++];
    memset(S, 0, sizeof(*S));
    S->n = n; S->rigid = 1; S->d = (real)d; S->visc_alpha = (real)visc_alpha; S->rho0 = (real)rho0;
    ALLOC3(S->pos, n); ALLOC3(S->vel, n); ALLOC3(S->svel, n); ALLOC3(S->force, n);
    ALLOC1(S->volume, n); ALLOC1(S->kerSumFromSelf, n);
    ALLOC1(S->mass, n); ALLOC1(S->VF_gamma, n); ALLOC1(S->VF_sphVolume, n); ALLOC1(S->VF_advVol, n);
    ALLOC1(S->VF_alpha, n); ALLOC1(S->VF_alpha2, n); ALLOC1(S->VF_kappa, n); ALLOC1(S->VF_kappaV, n);
    ALLOC1(S->VF_divdev, n);
    S->nnum = (int*)calloc((size_t)n + 1, sizeof(int));
    S->nidx = (PIdx*)calloc((size_t)n * s->P.cap + 1, sizeof(PIdx));
    S->ndis = (real*)calloc((size_t)n * s->P.cap + 1, sizeof(real));
    S->next = (PIdx*)calloc((size_t)n + 1, sizeof(PIdx));
    for (long i = 0; i < 3L * n; ++i) S->pos[i] = (real)xyz[i];
    if (prepare) prepare_solid_part_weight(s);
    return s->ns - 1;
}

/* Make solid k a dynamic rigid body (SphSolid(dynamic=true, RIGIDBODY),
 * SphBase.h:326): inner = its body-frame particle positions (3n), state = 25
 * doubles (transform[16] OpenGL column-major, com[3], linear[3],
 * angular[3]).  As SphWithBullet::addSolid does (SphWithBullet.cpp:
 * 131-135), the particles are placed at once and every solid's
 * kerSumFromSelf and volume recomputed (prepareSolidPartWeight). */
int orc_set_solid_dynamic(void* h, int k, const double* inner, const double* state) {
    OrcScene* s = (OrcScene*)h;
    if (k < 0 || k >= s->ns) return -1;
    OrcSolid* S = &s->S[k];
    if (!S->inner) ALLOC3(S->inner, S->n);
    for (long i = 0; i < 3L * S->n; ++i) S->inner[i] = (real)inner[i];
    S->dynamic = 1;
    solid_set_state(S, state);
    solid_update_particles(S);
    prepare_solid_part_weight(s);
    return 0;
}

void orc_set_rigid_callback(void* h, void* fn, void* user) {
    OrcScene* s = (OrcScene*)h;
    s->rigid_fn = (int (*)(void*, int, const int*, const double*, const double*, double, double*))fn;
    s->rigid_user = user;
}

/* rigidForceJoin of solid k about com (3 doubles); returns 0 */
int orc_rigid_force_join(void* h, int k, const double* com, double* force, double* torque) {
    OrcScene* s = (OrcScene*)h;
    if (k < 0 || k >= s->ns) return -1;
    real c[3] = {(real)com[0], (real)com[1], (real)com[2]}, tf[3], tt[3];
    rigid_force_join(&s->S[k], c, tf, tt);
    for (int i = 0; i < 3; ++i) { force[i] = tf[i]; torque[i] = tt[i]; }
    return 0;
}

int orc_rigid_error(void* h) { return ((OrcScene*)h)->rigid_err; }

int orc_add_fluid(void* h, int n, const double* xyz, const double* vel, double d, double rho0,
                  double visc_alpha, double tension) {
    OrcScene* s = (OrcScene*)h;
    if (s->nf >= 8) return -1;
    OrcFluid* F = &s->F[s->nf++];
    memset(F, 0, sizeof(*F));
    F->n = n; F->d = (real)d; F->rho0 = (real)rho0; F->visc_alpha = (real)visc_alpha; F->tension = (real)tension;
    ALLOC3(F->pos, n); ALLOC3(F->vel, n); ALLOC3(F->vel_adv, n); ALLOC3(F->acce_adv, n);
    ALLOC3(F->acceleration, n); ALLOC3(F->DFalpha1, n); ALLOC3(F->n_surf, n);
    ALLOC3(F->pos_pred, n); ALLOC3(F->acce_pressure, n); ALLOC3(F->dii, n); ALLOC3(F->sum_dijpj, n);
    ALLOC3(F->adv_vel, n); ALLOC3(F->acce_presure, n);
    ALLOC1(F->density, n); ALLOC1(F->DFalpha, n); ALLOC1(F->DFalpha2, n); ALLOC1(F->DFkappa, n);
    ALLOC1(F->DFkappaV, n); ALLOC1(F->density_adv, n); ALLOC1(F->divdev, n); ALLOC1(F->presure, n);
    ALLOC1(F->aii, n); ALLOC1(F->rho_adv, n); ALLOC1(F->p_l, n); ALLOC1(F->p_l2, n);
    F->beta = 1;
    ALLOC3(F->adv_acc, n); ALLOC3(F->VF_alpha1, n);
    ALLOC1(F->sphDensity, n); ALLOC1(F->VF_gamma, n); ALLOC1(F->VF_sphVolume, n); ALLOC1(F->VF_advVol, n);
    ALLOC1(F->VF_alpha, n); ALLOC1(F->VF_alpha2, n); ALLOC1(F->VF_kappa, n); ALLOC1(F->VF_kappaV, n);
    ALLOC1(F->VF_divdev, n);
    F->nnum = (int*)calloc((size_t)n + 1, sizeof(int));
    F->nidx = (PIdx*)calloc((size_t)n * s->P.cap + 1, sizeof(PIdx));
    F->ndis = (real*)calloc((size_t)n * s->P.cap + 1, sizeof(real));
    F->next = (PIdx*)calloc((size_t)n + 1, sizeof(PIdx));
    for (long i = 0; i < 3L * n; ++i) { F->pos[i] = (real)xyz[i]; F->vel[i] = vel ? (real)vel[i] : 0; }
    for (long i = 0; i < n; ++i) F->density[i] = (real)rho0; /* as the oracle harness of the reference */
    return s->nf - 1;
}

int orc_num_fluid(void* h, int k) { OrcScene* s = (OrcScene*)h; return k < s->nf ? s->F[k].n : -1; }
int orc_num_solid(void* h, int k) { OrcScene* s = (OrcScene*)h; return k < s->ns ? s->S[k].n : -1; }

int orc_stage(void* h, const char* name) {
    OrcScene* s = (OrcScene*)h;
    if (!strcmp(name, "neighbourSearch")) { neighbour_search(s, 1, 1, 0); return 0; }
    if (!strcmp(name, "prepareSolidPartWeight")) { prepare_solid_part_weight(s); return 0; }
    if (!strcmp(name, "updateSolidPartWeight")) { update_solid_part_weight(s); return 0; }
    if (!strcmp(name, "updateFluids")) { update_fluids(s, 0); return 0; }
    if (!strcmp(name, "DF_constantDensitySolverFirst")) { df_first(s); return 0; }
    if (!strcmp(name, "DF_constantDensitySolverSecond")) { df_second(s); return 0; }
    if (!strcmp(name, "DF_divergenceFreeSolver")) { df_divergence_free(s); return 0; }
    if (!strcmp(name, "DF_forceExceptPressure")) { df_force_except_pressure(s); return 0; }
    if (!strcmp(name, "df_step")) { df_step(s); return 0; }
    if (!strcmp(name, "updateSolids")) { update_solids(s); return 0; }
    if (!strcmp(name, "cfl_dt")) { cfl_dt(s); return 0; }
    if (!strcmp(name, "wc_computePressure")) { wc_pressure(s); return 0; }
    if (!strcmp(name, "wc_computeForce")) { wc_force(s); return 0; }
    if (!strcmp(name, "wc_step")) { wc_step(s); return 0; }
    if (orc_stage_iisph(s, name) == 0) return 0;
    return orc_stage_pci_ii(s, name);
}

static int fluid_field(OrcFluid* F, const char* f, real** p) {
#define V3(nm, arr) if (!strcmp(f, nm)) { *p = F->arr; return 3; }
#define V1(nm, arr) if (!strcmp(f, nm)) { *p = F->arr; return 1; }
    V3("position", pos) V3("velocity", vel) V3("vel_adv", vel_adv) V3("acce_adv", acce_adv)
    V3("acceleration", acceleration) V3("DFalpha1", DFalpha1) V3("n", n_surf)
    V3("pos_prediction", pos_pred) V3("acce_pressure", acce_pressure) V3("dii", dii)
    V3("sum_dijpj", sum_dijpj) V3("advectionVelocity", adv_vel) V3("acce_presure", acce_presure)
    V1("density", density) V1("DFalpha", DFalpha) V1("DFalpha2", DFalpha2) V1("DFkappa", DFkappa)
    V1("DFkappaV", DFkappaV) V1("density_adv", density_adv) V1("divergenceDeviation", divdev)
    V1("presure", presure) V1("aii", aii) V1("rho_adv", rho_adv) V1("p_l", p_l)
    V3("advectionAcceleration", adv_acc) V3("VF_alpha1", VF_alpha1) V1("sphDensity", sphDensity)
    V1("VF_gamma", VF_gamma) V1("VF_sphVolume", VF_sphVolume) V1("VF_advectionVolume", VF_advVol)
    V1("VF_alpha", VF_alpha) V1("VF_alpha2", VF_alpha2) V1("VF_kappa", VF_kappa) V1("VF_kappaV", VF_kappaV)
    V1("VF_divergenceDeviation", VF_divdev)
#undef V3
#undef V1
    return -1;
}

int orc_get(void* h, int k, const char* field, double* out) {
    OrcScene* s = (OrcScene*)h;
    real* p; int c = fluid_field(&s->F[k], field, &p);
    if (c < 0) return -1;
    for (long i = 0; i < (long)c * s->F[k].n; ++i) out[i] = (double)p[i];
    return 0;
}
int orc_set(void* h, int k, const char* field, const double* in) {
    OrcScene* s = (OrcScene*)h;
    real* p; int c = fluid_field(&s->F[k], field, &p);
    if (c < 0) return -1;
    for (long i = 0; i < (long)c * s->F[k].n; ++i) p[i] = (real)in[i];
    return 0;
}
int orc_get_solid(void* h, int k, const char* field, double* out) {
    OrcScene* s = (OrcScene*)h;
    OrcSolid* S = &s->S[k];
    real* p = 0; int c = 0;
    if (!strcmp(field, "position")) { p = S->pos; c = 3; }
    else if (!strcmp(field, "velocity")) { p = S->vel; c = 3; }
    else if (!strcmp(field, "singleVelocity")) { p = S->svel; c = 3; }
    else if (!strcmp(field, "force")) { p = S->force; c = 3; }
    else if (!strcmp(field, "volume")) { p = S->volume; c = 1; }
    else if (!strcmp(field, "kerSumFromSelf")) { p = S->kerSumFromSelf; c = 1; }
    else if (!strcmp(field, "mass")) { p = S->mass; c = 1; }
    else if (!strcmp(field, "VF_gamma")) { p = S->VF_gamma; c = 1; }
    else if (!strcmp(field, "VF_sphVolume")) { p = S->VF_sphVolume; c = 1; }
    else if (!strcmp(field, "VF_advectionVolume")) { p = S->VF_advVol; c = 1; }
    else if (!strcmp(field, "VF_alpha")) { p = S->VF_alpha; c = 1; }
    else if (!strcmp(field, "VF_alpha2")) { p = S->VF_alpha2; c = 1; }
    else if (!strcmp(field, "VF_kappa")) { p = S->VF_kappa; c = 1; }
    else if (!strcmp(field, "VF_kappaV")) { p = S->VF_kappaV; c = 1; }
    else if (!strcmp(field, "VF_divergenceDeviation")) { p = S->VF_divdev; c = 1; }
    else return -1;
    for (long i = 0; i < (long)c * S->n; ++i) out[i] = (double)p[i];
    return 0;
}
int orc_set_solid(void* h, int k, const char* field, const double* in) {
    OrcScene* s = (OrcScene*)h;
    OrcSolid* S = &s->S[k];
    real* p = 0; int c = 0;
    if (!strcmp(field, "volume")) { p = S->volume; c = 1; }
    else if (!strcmp(field, "kerSumFromSelf")) { p = S->kerSumFromSelf; c = 1; }
    else if (!strcmp(field, "velocity")) { p = S->vel; c = 3; }
    else return -1;
    for (long i = 0; i < (long)c * S->n; ++i) p[i] = (real)in[i];
    return 0;
}

int orc_neighbours(void* h, int kind, int k, int* counts, int* t, int* idx, double* dis) {
    OrcScene* s = (OrcScene*)h;
    const int cap = s->P.cap;
    int n = kind == 0 ? s->F[k].n : s->S[k].n;
    const int* nn = kind == 0 ? s->F[k].nnum : s->S[k].nnum;
    const PIdx* L = kind == 0 ? s->F[k].nidx : s->S[k].nidx;
    const real* D = kind == 0 ? s->F[k].ndis : s->S[k].ndis;
    for (long i = 0; i < n; ++i) {
        counts[i] = nn[i];
        for (int j = 0; j < nn[i]; ++j) {
            t[i * cap + j] = L[i * cap + j].t;
            idx[i * cap + j] = L[i * cap + j].i;
            dis[i * cap + j] = (double)D[i * cap + j];
        }
    }
    return cap;
}

int orc_cells(void* h, int kind, int k, long long* cell) {
    OrcScene* s = (OrcScene*)h;
    if (!s->gridFirst) grid_setup(s);
    int n = kind == 0 ? s->F[k].n : s->S[k].n;
    const real* P = kind == 0 ? s->F[k].pos : s->S[k].pos;
    for (long i = 0; i < n; ++i) cell[i] = grid_of_pos(s, P + 3 * i);
    return 0;
}

void orc_grid_info(void* h, double* min3, double* divisor, long long* num3) {
    OrcScene* s = (OrcScene*)h;
    if (!s->gridFirst) grid_setup(s);
    for (int i = 0; i < 3; ++i) { min3[i] = s->gmin[i]; num3[i] = s->gnum[i]; }
    *divisor = s->divisor;
}

void orc_error_counts(void* h, long long* zeroDis, long long* tooMany) {
    OrcScene* s = (OrcScene*)h;
    *zeroDis = s->zeroDis; *tooMany = s->tooMany;
}

void orc_stats(void* h, int* iters, double* errs, double* dt, int* frame) {
    OrcScene* s = (OrcScene*)h;
    iters[0] = s->it_density; iters[1] = s->it_div; iters[2] = s->it_pci; iters[3] = s->it_ii;
    errs[0] = s->err_density; errs[1] = s->err_div; errs[2] = s->err_pci; errs[3] = s->err_ii;
    *dt = s->P.dt; *frame = s->frame;
}

/* IISph (volume form): iterations and errors of the last divergence-free and
 * constant-volume loops (summed over phases) */
void orc_vf_stats(void* h, int* iters, double* errs) {
    OrcScene* s = (OrcScene*)h;
    iters[0] = s->it_iv_div; iters[1] = s->it_iv_cv;
    errs[0] = s->err_iv_div; errs[1] = s->err_iv_cv;
}

void orc_set_dt(void* h, double dt) { ((OrcScene*)h)->P.dt = dt; }
double orc_pci_delta(void* h) { return (double)((OrcScene*)h)->pci_delta; }
void orc_set_frame(void* h, int f) { ((OrcScene*)h)->frame = f; }

double orc_kernel(void* h, int grad, double r) {
    OrcScene* s = (OrcScene*)h;
    return grad ? (double)ker_W_grad(s, (real)r) : (double)ker_W(s, (real)r);
}

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
