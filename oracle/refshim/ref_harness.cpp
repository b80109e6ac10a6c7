/* C entry points around the reference's own solver classes (test
 * infrastructure: the oracle build of the reference, compiled by
 * oracle/build_ref.py into oracle/_ref/libref_<solver>[_f64].so).
 *
 * The harness derives from one reference solver class (REF_SOLVER_CLASS, e.g.
 * DFSPH from DFSPH.h:10) with empty setupScene()/stepEvent(), fills
 * m_Fluids / m_Solids directly (the reference builds them in
 * SphWithIO::addFluidCuboid, SphWithIO.cpp:149-194, and addRigidCuboid,
 * SphWithIO.cpp:642-659), and exposes the reference's own stage functions by
 * name so that tests can run "given state S, call stage X, read field F".
 *
 * Kernel constants: the reference never calls ker_update_numbers()
 * (SphBase.h:808-829; the call at SphBase.cpp:853 is commented out), so every
 * single-argument ker_W / ker_W_grad would use m_ker_h = -1.  The harness calls
 * it once the parameters are set, which gives m_ker_h = smoothRadius_h / 2, the
 * intended value.
 *
 * All field transfers are in double so the float and double builds share one
 * interface; float inputs round-trip exactly. */
#include <cstring>
#include <string>
#include <unistd.h>
#include REF_SOLVER_HEADER

#ifdef REF_TAG_dfsph_capped
int ref_df_iter_count[2];  // written by the capped DFSPH loops
#endif

extern "C" {
struct RefParams {
    double spacing_r, smoothRadius_h, dt;
    double gravity[3];
    double densityErro_eta, soundSpeed_cs;
    double nu;               /* m_TH.nu (viscosity of the DFSPH/IISPH_M force loops) */
    double th_h, th_r, th_bt; /* m_TH.h / r / bt (WCSPH surface tension, adhesion) */
    double spaceMin[3], spaceMax[3];
    /* m_TH.enable_vortex / alpha / zeta / nu_t (DFSPH's vorticity options) */
    int enable_vortex;
    double alpha, zeta, nu_t;
};
}

class RefHarness : public REF_SOLVER_CLASS {
public:
    void setupScene() override {}
    void stepEvent() override {}

    void apply(const RefParams& p) {
        m_TH.spacing_r = real_t(p.spacing_r);
        m_TH.smoothRadius_h = real_t(p.smoothRadius_h);
        m_TH.dt = real_t(p.dt);
        m_TH.gravity_g = vec_t(real_t(p.gravity[0]), real_t(p.gravity[1]), real_t(p.gravity[2]));
        m_TH.densityErro_eta = real_t(p.densityErro_eta);
        m_TH.soundSpeed_cs = real_t(p.soundSpeed_cs);
        m_TH.nu = real_t(p.nu);
        m_TH.h = real_t(p.th_h);
        m_TH.r = real_t(p.th_r);
        m_TH.bt = real_t(p.th_bt);
        m_TH.spaceMin = vec_t(real_t(p.spaceMin[0]), real_t(p.spaceMin[1]), real_t(p.spaceMin[2]));
        m_TH.spaceMax = vec_t(real_t(p.spaceMax[0]), real_t(p.spaceMax[1]), real_t(p.spaceMax[2]));
        m_TH.enable_vortex = p.enable_vortex;
        m_TH.alpha = real_t(p.alpha);
        m_TH.zeta = real_t(p.zeta);
        m_TH.nu_t = real_t(p.nu_t);
        ker_update_numbers();
#ifdef REF_TAG_pcisph
        /* PciSph() leaves the pci_updateDelta cache keys uninitialised
         * (PciSph.h:35,63); start from values that force the computation. */
        pci_last_dt = pci_last_sp = pci_last_h = real_t(-1);
#endif
#ifdef REF_TAG_iisph
        /* IISph: the temperature / melting update (SphBase::updateTemperature,
         * run by IISph::sphStep when m_TH.phaseTransition, IISph.cpp:74-76)
         * is off, as in the reference's own demo scene (Demo-mySPH.h:49). */
        m_TH.phaseTransition = false;
        m_TH.dF_iteration = m_TH.cV_iteration = 0;  // uninitialised members (SphBase.h)
#endif
    }

    int stage(const std::string& s) {
        if (s == "neighbourSearch") { neighbourSearch(); return 0; }
        if (s == "prepareSolidPartWeight") { prepareSolidPartWeight(); return 0; }
        if (s == "updateSolidPartWeight") { updateSolidPartWeight(); return 0; }
        if (s == "updateFluids") { updateFluids(); return 0; }
        if (s == "sphStep") { sphStep(); return 0; }
        if (s == "runOneStep") { runOneStep(); return 0; }
        if (s == "updateSolids") { updateSolids(); return 0; }
#if defined(REF_TAG_dfsph) || defined(REF_TAG_dfsph_capped)
        if (s == "DF_constantDensitySolverFirst") { DF_constantDensitySolverFirst(); return 0; }
        if (s == "DF_constantDensitySolverSecond") { DF_constantDensitySolverSecond(); return 0; }
        if (s == "DF_divergenceFreeSolver") { DF_divergenceFreeSolver(); return 0; }
        if (s == "DF_forceExceptPressure") { DF_forceExceptPressure(); return 0; }
#endif
#ifdef REF_TAG_wcsph
        if (s == "wc_computePressure") { wc_computePressure(); return 0; }
        if (s == "wc_computeForce") { wc_computeForce(); return 0; }
#endif
#ifdef REF_TAG_pcisph
        if (s == "pci_computeForce") { pci_computeForce(); return 0; }
#endif
#ifdef REF_TAG_iisphm
        if (s == "ii_computePressure") { ii_computePressure(); return 0; }
        if (s == "ii_computeForcePressure") { ii_computeForcePressure(); return 0; }
#endif
#ifdef REF_TAG_iisph
        if (s == "DF_prepareAttribute") { DF_prepareAttribute(); return 0; }
        if (s == "VF_prepareAttribute") { VF_prepareAttribute(); return 0; }
        if (s == "advectionStep") { advectionStep(); return 0; }
        if (s == "VF_divergenceFreeSolver") { VF_divergenceFreeSolver(); return 0; }
        if (s == "VF_constantVolumeSolver") { VF_constantVolumeSolver(); return 0; }
#endif
        return -1;
    }

    /* field accessors: returns component count, or -1 if unknown */
    static int fluidField(FluidPart& p, const char* f, real_t** ptr) {
#define SCAL(name) if (!strcmp(f, #name)) { *ptr = &p.name; return 1; }
#define VEC(name) if (!strcmp(f, #name)) { *ptr = &p.name[0]; return 3; }
        VEC(position) VEC(velocity) VEC(advectionVelocity) VEC(advectionAcceleration)
        VEC(acce_presure) VEC(dii) VEC(sum_dijpj) VEC(n) VEC(acceleration)
        VEC(DFalpha1) VEC(vel_adv) VEC(acce_adv) VEC(omega) VEC(angular_velocity) VEC(dOmega)
        VEC(n0Vorticity) VEC(deltaVorticity) VEC(psi) VEC(vorticity)
        SCAL(aii) SCAL(rho_adv) SCAL(p_l) SCAL(d) SCAL(sphDensity) SCAL(advectionDensity)
        SCAL(restDensity) SCAL(presure) SCAL(mass) SCAL(density) SCAL(density_adv)
        SCAL(DFalpha) SCAL(DFalpha2) SCAL(DFkappa) SCAL(DFkappaV) SCAL(divergenceDeviation)
        SCAL(restVolume) SCAL(beta) SCAL(kinematicViscosity) SCAL(temperature) SCAL(temperatureNext)
        SCAL(DF_alpha) SCAL(DF_alpha2) SCAL(VF_gamma) SCAL(VF_sphVolume) SCAL(VF_advectionVolume)
        SCAL(VF_alpha) SCAL(VF_alpha2) SCAL(VF_kappa) SCAL(VF_kappaV) SCAL(VF_divergenceDeviation)
        VEC(DF_alpha1) VEC(VF_alpha1)
#ifdef PREDICTION_PCISPH
        VEC(acce_pressure) VEC(pos_prediction)
#endif
        return -1;
    }
    static int solidField(BoundPart& p, const char* f, real_t** ptr) {
        VEC(position) VEC(velocity) VEC(force) VEC(singleVelocity)
        SCAL(volume) SCAL(kerSumFromSelf) SCAL(d) SCAL(restDensity) SCAL(sphDensity)
        SCAL(mass) SCAL(kinematicViscosity) SCAL(DF_alpha) SCAL(VF_gamma) SCAL(VF_sphVolume)
        SCAL(VF_advectionVolume) SCAL(VF_alpha) SCAL(VF_alpha2) SCAL(VF_kappa) SCAL(VF_kappaV)
        SCAL(VF_divergenceDeviation)
        return -1;
#undef SCAL
#undef VEC
    }

    // ---- C-callable bodies (members, so friend access to SphBase applies) ----
    static void* ref_create_impl(const RefParams* p, const char* logdir) {
        /* SphBase::SphBase opens a date-named log file in the working directory
         * (SphBase.cpp:228-237); construct inside logdir so it lands there. */
        char cwd[4096];
        if (!getcwd(cwd, sizeof cwd)) cwd[0] = 0;
        if (logdir && logdir[0] && chdir(logdir) != 0) return nullptr;
        RefHarness* h = new RefHarness();
        if (cwd[0] && chdir(cwd) != 0) { delete h; return nullptr; }
        h->apply(*p);
        return h;
    }

    static void ref_destroy_impl(void* h) { delete static_cast<RefHarness*>(h); }

    static void ref_set_params_impl(void* hh, const RefParams* p) { static_cast<RefHarness*>(hh)->apply(*p); }

    static int ref_threads_impl(void) { return omp_get_max_threads(); }

    /* A static rigid solid (SphSolid(false, RIGIDBODY, ...), SphBase.h:326) whose
     * boundary particles sit at xyz; prepareSolidPartWeight() (SphBase.cpp:766)
     * then computes kerSumFromSelf and volume, as SphWithBullet::addSolid does. */
    static int ref_add_solid_impl(void* hh, int n, const double* xyz, double d, double visc_alpha,
                      double restDensity, int prepare) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        SphSolid s(false, SphSolid::RIGIDBODY, static_cast<real_t>(visc_alpha), 0);
        BoundaryParticle b = BoundaryParticle();
        b.d = real_t(d);
        b.restDensity = real_t(restDensity);
        for (int i = 0; i < n; ++i) {
            b.position = vec_t(real_t(xyz[3 * i]), real_t(xyz[3 * i + 1]), real_t(xyz[3 * i + 2]));
            s.boundaryParticles.push_back(b);
            s.innerPositions.push_back(b.position);
        }
        h->m_Solids.push_back(s);
        if (prepare) h->prepareSolidPartWeight();
        return int(h->m_Solids.size()) - 1;
    }

    /* A new fluid phase (as addFluidCuboid(newFluid=true, ...) creates one,
     * SphWithIO.cpp:167) holding n particles. */
    static int ref_add_fluid_impl(void* hh, int n, const double* xyz, const double* vel, double d,
                      double rho0, double visc_alpha, double tension) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        SphFluid f(static_cast<real_t>(rho0), static_cast<real_t>(visc_alpha), static_cast<real_t>(tension));
        FluidParticle p = FluidParticle();
        p.d = real_t(d);
        p.restDensity = real_t(rho0);
        /* IISph reads beta (restDensity = rho0 * beta, IISph.cpp:109-110) and the
         * temperature; a value-initialised particle has beta = 0.  The
         * reference's demo scene sets beta = 1 at 0 degrees C
         * (Demo-mySPH.h:90-93). */
        p.beta = real_t(1);
        p.temperature = p.temperatureNext = real_t(273.15);
        /* WcSph::wc_computePressure reads the neighbours' density before it is
         * first computed (WcSph.cpp:131, for the surface normal); start from
         * the rest density so that read is finite. */
        p.density = real_t(rho0);
        for (int i = 0; i < n; ++i) {
            p.position = vec_t(real_t(xyz[3 * i]), real_t(xyz[3 * i + 1]), real_t(xyz[3 * i + 2]));
            p.velocity = vel ? vec_t(real_t(vel[3 * i]), real_t(vel[3 * i + 1]), real_t(vel[3 * i + 2]))
                             : vec_t(0);
            f.fluidParticles.push_back(p);
        }
        h->m_Fluids.push_back(f);
        return int(h->m_Fluids.size()) - 1;
    }

    static int ref_num_fluid_impl(void* hh, int k) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        return (k < 0 || k >= int(h->m_Fluids.size())) ? -1 : int(h->m_Fluids[k].fluidParticles.size());
    }
    static int ref_num_solid_impl(void* hh, int k) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        return (k < 0 || k >= int(h->m_Solids.size())) ? -1 : int(h->m_Solids[k].boundaryParticles.size());
    }

    static int ref_stage_impl(void* hh, const char* name) { return static_cast<RefHarness*>(hh)->stage(name); }

    static int ref_get_impl(void* hh, int k, const char* field, double* out) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        auto& v = h->m_Fluids[k].fluidParticles;
        for (size_t i = 0; i < v.size(); ++i) {
            real_t* p; int c = RefHarness::fluidField(v[i], field, &p);
            if (c < 0) return -1;
            for (int j = 0; j < c; ++j) out[i * c + j] = double(p[j]);
        }
        return 0;
    }
    static int ref_set_impl(void* hh, int k, const char* field, const double* in) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        auto& v = h->m_Fluids[k].fluidParticles;
        for (size_t i = 0; i < v.size(); ++i) {
            real_t* p; int c = RefHarness::fluidField(v[i], field, &p);
            if (c < 0) return -1;
            for (int j = 0; j < c; ++j) p[j] = real_t(in[i * c + j]);
        }
        return 0;
    }
    static int ref_get_solid_impl(void* hh, int k, const char* field, double* out) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        auto& v = h->m_Solids[k].boundaryParticles;
        for (size_t i = 0; i < v.size(); ++i) {
            real_t* p; int c = RefHarness::solidField(v[i], field, &p);
            if (c < 0) return -1;
            for (int j = 0; j < c; ++j) out[i * c + j] = double(p[j]);
        }
        return 0;
    }

    /* Neighbour lists of fluid phase k (kind 0) or solid k (kind 1): per particle
     * the count and up to NeigbStr::maxNeigbNum (PartIdx t, i, dis) entries in
     * list order (SphBase.h:620-646). */
    static int ref_neighbours_impl(void* hh, int kind, int k, int* counts, int* t, int* idx, double* dis) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        const auto& L = kind == 0 ? h->mg_NeigbOfFluids[k] : h->mg_NeigbOfSolids[k];
        const int cap = SphBase::NeigbStr::maxNeigbNum;
        for (size_t i = 0; i < L.size(); ++i) {
            counts[i] = L[i].num;
            for (int j = 0; j < L[i].num; ++j) {
                t[i * cap + j] = L[i].neigs[j].pidx.t;
                idx[i * cap + j] = L[i].neigs[j].pidx.i;
                dis[i * cap + j] = double(L[i].neigs[j].dis);
            }
        }
        return cap;
    }

    /* Grid cell index (SpaceGridStruct::gridOfPos, SphBase.h:700-701) of every
     * particle of fluid phase k (kind 0) or solid k (kind 1). */
    static int ref_cells_impl(void* hh, int kind, int k, long long* cell) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        if (kind == 0) {
            auto& v = h->m_Fluids[k].fluidParticles;
            for (size_t i = 0; i < v.size(); ++i) cell[i] = (long long)h->mg_NS.gridOfPos(v[i].position);
        } else {
            auto& v = h->m_Solids[k].boundaryParticles;
            for (size_t i = 0; i < v.size(); ++i) cell[i] = (long long)h->mg_NS.gridOfPos(v[i].position);
        }
        return 0;
    }

    static void ref_grid_info_impl(void* hh, double* min3, double* divisor, long long* num3) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        for (int i = 0; i < 3; ++i) { min3[i] = double(h->mg_NS.min[i]); num3[i] = (long long)h->mg_NS.num[i]; }
        *divisor = double(h->mg_NS.divisor);
    }

    static void ref_error_counts_impl(void* hh, int* zeroDis, int* tooMany) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        *zeroDis = h->m_EC.zeroDis;
        *tooMany = h->m_EC.tooManyNeigb;
    }

    static void ref_set_dt_impl(void* hh, double dt) { static_cast<RefHarness*>(hh)->m_TH.dt = real_t(dt); }
    static int ref_frame_impl(void* hh) { return static_cast<RefHarness*>(hh)->m_TH.frameNumber; }
    static void ref_set_frame_impl(void* hh, int f) { static_cast<RefHarness*>(hh)->m_TH.frameNumber = f; }
    /* PCISPH loop bounds m_minIterations / m_maxIterations (PciSph.h:35);
     * returns -1 for the other solvers */
    static int ref_set_iter_limits_impl(void* hh, int mn, int mx) {
#ifdef REF_TAG_pcisph
        RefHarness* h = static_cast<RefHarness*>(hh);
        h->m_minIterations = mn;
        h->m_maxIterations = mx;
        return 0;
#else
        (void)hh; (void)mn; (void)mx;
        return -1;
#endif
    }
    /* IISph iteration counters m_TH.dF_iteration / cV_iteration (each loop
     * adds its iterations - 1, IISph.cpp:1449, 794); read and reset.
     * Returns -1 for the other solvers. */
    static int ref_vf_iters_impl(void* hh, int* df, int* cv) {
#ifdef REF_TAG_iisph
        RefHarness* h = static_cast<RefHarness*>(hh);
        *df = int(h->m_TH.dF_iteration);
        *cv = int(h->m_TH.cV_iteration);
        h->m_TH.dF_iteration = 0;
        h->m_TH.cV_iteration = 0;
        return 0;
#else
        (void)hh; *df = *cv = 0;
        return -1;
#endif
    }
    /* DFSPH "capped" build: density and divergence loop iterations summed
     * since the last call (counted on the loops' closing lines by
     * build_ref.py's edit of the copy); read and reset.  Returns -1 for the
     * other builds. */
    static int ref_df_iters_impl(int* dens, int* div) {
#ifdef REF_TAG_dfsph_capped
        *dens = ref_df_iter_count[0];
        *div = ref_df_iter_count[1];
        ref_df_iter_count[0] = ref_df_iter_count[1] = 0;
        return 0;
#else
        *dens = *div = 0;
        return -1;
#endif
    }
    static int ref_set_solid_impl(void* hh, int k, const char* field, const double* in) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        auto& v = h->m_Solids[k].boundaryParticles;
        for (size_t i = 0; i < v.size(); ++i) {
            real_t* p; int c = RefHarness::solidField(v[i], field, &p);
            if (c < 0) return -1;
            for (int j = 0; j < c; ++j) p[j] = real_t(in[i * c + j]);
        }
        return 0;
    }
    /* Dynamic rigid solid k (SphSolid::dynamic, SphBase.h:330) with body-frame
     * positions inner (3n doubles, SphSolid::innerPositions) and initial
     * state (25 doubles, see SphWithIO.h); placed at once, then
     * prepareSolidPartWeight() recomputes every solid's kerSumFromSelf and
     * volume, as SphWithBullet::addSolid does (SphWithBullet.cpp:131-135). */
    static int ref_set_solid_dynamic_impl(void* hh, int k, const double* inner, const double* state) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        if (k < 0 || k >= int(h->m_Solids.size())) return -1;
        SphSolid& s = h->m_Solids[k];
        s.dynamic = true;
        s.type = SphSolid::RIGIDBODY;
        s.innerPositions.resize(s.boundaryParticles.size());
        for (size_t i = 0; i < s.innerPositions.size(); ++i)
            s.innerPositions[i] = vec_t(real_t(inner[3 * i]), real_t(inner[3 * i + 1]), real_t(inner[3 * i + 2]));
        h->setRigidState(k, state);
        h->placeSolid(k);
        h->prepareSolidPartWeight();
        return 0;
    }
    static void ref_set_rigid_callback_impl(void* hh, void* fn, void* user) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        h->rigid_fn = reinterpret_cast<RigidFn>(fn);
        h->rigid_user = user;
    }
    static int ref_rigid_error_impl(void* hh) { return static_cast<RefHarness*>(hh)->rigid_err; }
    /* SphSolid::rigidForceJoin of solid k about com (SphBase.cpp:131-143) */
    static int ref_rigid_force_join_impl(void* hh, int k, const double* com, double* force, double* torque) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        if (k < 0 || k >= int(h->m_Solids.size())) return -1;
        vec_t f;
        vec3_t t;
        h->m_Solids[k].rigidForceJoin(vec_t(real_t(com[0]), real_t(com[1]), real_t(com[2])), f, t);
        for (int c = 0; c < 3; ++c) { force[c] = double(f[c]); torque[c] = double(t[c]); }
        return 0;
    }
    static double ref_kernel_impl(void* hh, int grad, double r) {
        RefHarness* h = static_cast<RefHarness*>(hh);
        return grad ? double(h->ker_W_grad(real_t(r))) : double(h->ker_W(real_t(r)));
    }


};



extern "C" {
void* ref_create(const RefParams* p, const char* logdir) { return RefHarness::ref_create_impl(p, logdir); }
void ref_destroy(void* h) { RefHarness::ref_destroy_impl(h); }
void ref_set_params(void* hh, const RefParams* p) { RefHarness::ref_set_params_impl(hh, p); }
int ref_threads(void) { return RefHarness::ref_threads_impl(); }
int ref_add_solid(void* hh, int n, const double* xyz, double d, double visc_alpha,
                  double restDensity, int prepare) { return RefHarness::ref_add_solid_impl(hh, n, xyz, d, visc_alpha, restDensity, prepare); }
int ref_add_fluid(void* hh, int n, const double* xyz, const double* vel, double d,
                  double rho0, double visc_alpha, double tension) { return RefHarness::ref_add_fluid_impl(hh, n, xyz, vel, d, rho0, visc_alpha, tension); }
int ref_num_fluid(void* hh, int k) { return RefHarness::ref_num_fluid_impl(hh, k); }
int ref_num_solid(void* hh, int k) { return RefHarness::ref_num_solid_impl(hh, k); }
int ref_stage(void* hh, const char* name) { return RefHarness::ref_stage_impl(hh, name); }
int ref_get(void* hh, int k, const char* field, double* out) { return RefHarness::ref_get_impl(hh, k, field, out); }
int ref_set(void* hh, int k, const char* field, const double* in) { return RefHarness::ref_set_impl(hh, k, field, in); }
int ref_get_solid(void* hh, int k, const char* field, double* out) { return RefHarness::ref_get_solid_impl(hh, k, field, out); }
int ref_neighbours(void* hh, int kind, int k, int* counts, int* t, int* idx, double* dis) { return RefHarness::ref_neighbours_impl(hh, kind, k, counts, t, idx, dis); }
int ref_cells(void* hh, int kind, int k, long long* cell) { return RefHarness::ref_cells_impl(hh, kind, k, cell); }
void ref_grid_info(void* hh, double* min3, double* divisor, long long* num3) { RefHarness::ref_grid_info_impl(hh, min3, divisor, num3); }
void ref_error_counts(void* hh, int* zeroDis, int* tooMany) { RefHarness::ref_error_counts_impl(hh, zeroDis, tooMany); }
void ref_set_dt(void* hh, double dt) { RefHarness::ref_set_dt_impl(hh, dt); }
int ref_frame(void* hh) { return RefHarness::ref_frame_impl(hh); }
void ref_set_frame(void* hh, int f) { RefHarness::ref_set_frame_impl(hh, f); }
double ref_kernel(void* hh, int grad, double r) { return RefHarness::ref_kernel_impl(hh, grad, r); }
int ref_set_iter_limits(void* hh, int mn, int mx) { return RefHarness::ref_set_iter_limits_impl(hh, mn, mx); }
int ref_vf_iters(void* hh, int* df, int* cv) { return RefHarness::ref_vf_iters_impl(hh, df, cv); }
int ref_df_iters(int* dens, int* div) { return RefHarness::ref_df_iters_impl(dens, div); }
int ref_set_solid(void* hh, int k, const char* field, const double* in) { return RefHarness::ref_set_solid_impl(hh, k, field, in); }
/* SphBase::SphBase sets the OpenMP thread count to omp_get_num_procs()
 * (SphBase.cpp:242-243); this overrides it (1 thread makes the racy loops of
 * IISph_M.cpp:315-351 deterministic) */
void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_set_solid_dynamic(void* hh, int k, const double* inner, const double* state) {
    return RefHarness::ref_set_solid_dynamic_impl(hh, k, inner, state);
}
void ref_set_rigid_callback(void* hh, void* fn, void* user) { RefHarness::ref_set_rigid_callback_impl(hh, fn, user); }
int ref_rigid_error(void* hh) { return RefHarness::ref_rigid_error_impl(hh); }
int ref_rigid_force_join(void* hh, int k, const double* com, double* force, double* torque) {
    return RefHarness::ref_rigid_force_join_impl(hh, k, com, force, torque);
}
}  // extern "C"
