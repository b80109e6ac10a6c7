/*
 * sphgpu_solver.hpp -- C++ drop-in for the reference's solver classes.
 *
 * GpuSolver<Base, Solver> derives from one of the reference's solver classes
 * (WcSph, PciSph, IISph_M, IISph, DFSPH; WcSph.h:24, PciSph.h:31,
 * IISph_M.h:10, IISph.h:10, DFSPH.h:10) and
 * overrides its step, virtual void sphStep() (SphBase.h:420), with one call
 * into the C ABI of include/sphgpu.h.  A reference scene switches to the GPU
 * by changing its base class:
 *
 *     class mySPH : public DFSPH                           // CPU (reference)
 *     class mySPH : public GpuSolver<DFSPH, SPHGPU_DFSPH>  // GPU (sm_100a)
 *
 * setupScene(), stepEvent(), runOneStep() (SphBase.cpp:348-354) and the
 * particle arrays m_Fluids / m_Solids (SphBase.h:660-661) keep their meaning:
 * before the first step the scene is uploaded (walls as static solids, one
 * phase per SphFluid); after every step positions, velocities and densities
 * (IISph: sphDensity) are written back into m_Fluids[k].fluidParticles,
 * with particles that left
 * [spaceMin, spaceMax] removed as SphFluid::removeOutsideParts does
 * (SphBase.cpp:26-48).  If stepEvent() changes the number of particles of a
 * phase, the scene is uploaded again before the next step.  m_EC receives
 * the step's zero-distance and neighbour-overflow counts (SphBase.h:586-602).
 *
 * Dynamic rigid solids (SphSolid::dynamic, SphBase.h:330; DFSPH): uploaded
 * with their innerPositions and the state gpuRigidState() gives; every step
 * the library calls gpuRigidStep() with each dynamic solid's joined force
 * and torque -- the exchange SphWithBullet::updateSolids has with Bullet
 * (SphWithBullet.cpp:180-224, 302-317) -- and after the step the solids'
 * boundaryParticles positions and velocities are written back.
 *
 * Header only; needs the reference's class declarations included first and
 * links against libsphgpu.so.
 */
#ifndef SPHGPU_SOLVER_HPP_
#define SPHGPU_SOLVER_HPP_

#include <stdexcept>
#include <string>
#include <vector>

#include "sphgpu.h"

template <class Base, int Solver>
class GpuSolver : public Base {
public:
    GpuSolver() { sphgpu_params_default(&gpu_params_); }
    ~GpuSolver() override {
        if (gpu_) sphgpu_destroy(gpu_);
    }

    /* Solver controls that m_TH does not hold (loop goals and caps, CFL,
     * neighbour cap); defaults are sphgpu_params_default()'s.  Changes take
     * effect at the next upload. */
    SphParams& gpuParams() { return gpu_params_; }
    /* Statistics of the last step (iterations, errors, dt, status). */
    const SphStepStats& gpuStats() const { return stats_; }
    /* CUDA device the scene runs on (set before the first step). */
    void setGpuDevice(int d) { device_ = d; }

    /* Rigid-body world of the dynamic solids.  gpuRigidState(k): solid k's
     * state at upload; the default is the identity transform (its
     * innerPositions are its positions under the identity, SphBase.h:
     * 334-336) with the centre of mass at the particles' centroid, at rest.
     * gpuRigidStep: apply force[3i..] and torque[3i..] to solid solids[i],
     * advance the bodies by dt, write their new states into states[i] (which
     * hold the current ones); the default keeps them.  A scene with Bullet
     * overrides both with SphWithBullet.cpp:185-210's calls
     * (applyCentralForce, applyTorque, stepSimulation, getOpenGLMatrix,
     * getCenterOfMassPosition, getLinearVelocity, getAngularVelocity). */
    virtual SphRigidState gpuRigidState(int solid) {
        SphRigidState st = {};
        st.transform[0] = st.transform[5] = st.transform[10] = st.transform[15] = 1.f;
        const auto& in = this->m_Solids[solid].innerPositions;
        double c[3] = {0, 0, 0};
        for (auto& x : in)
            for (int k = 0; k < 3; ++k) c[k] += x[k];
        for (int k = 0; k < 3; ++k) st.center_of_mass[k] = in.empty() ? 0.f : (float)(c[k] / in.size());
        return st;
    }
    virtual void gpuRigidStep(int n, const int* solids, const double* force, const double* torque, double dt,
                              SphRigidState* states) {
        (void)n; (void)solids; (void)force; (void)torque; (void)dt; (void)states;
    }

protected:
    void sphStep() override {
        if (!gpu_ || host_layout_changed()) upload();
        int rc = sphgpu_step(gpu_, Solver, 1, &stats_);
        if (rc < 0 && rc != SPHGPU_EMAXITER) fail("sphgpu_step", rc);
        this->m_EC.zeroDis += stats_.zero_distance;
        this->m_EC.tooManyNeigb += stats_.neighbour_overflow;
        download();
        download_solids();
    }

private:
    sphgpu_t gpu_ = nullptr;
    SphParams gpu_params_;
    SphStepStats stats_ = {};
    int device_ = 0;
    std::vector<size_t> counts_;  // per phase, as last written to m_Fluids

    static int rigid_trampoline(void* user, int n, const int* solids, const double* force, const double* torque,
                                double dt, SphRigidState* states) {
        try {
            static_cast<GpuSolver*>(user)->gpuRigidStep(n, solids, force, torque, dt, states);
            return 0;
        } catch (...) {
            return 1;  // the step call then fails with SPHGPU_EINVAL
        }
    }

    void fail(const char* what, int rc) {
        char buf[512] = {0};
        if (gpu_) sphgpu_last_error(gpu_, buf, sizeof buf);
        throw std::runtime_error(std::string(what) + " failed (" + std::to_string(rc) + "): " + buf);
    }

    bool host_layout_changed() const {
        if (counts_.size() != this->m_Fluids.size()) return true;
        for (size_t k = 0; k < counts_.size(); ++k)
            if (counts_[k] != this->m_Fluids[k].fluidParticles.size()) return true;
        return false;
    }

    void upload() {
        if (gpu_) { sphgpu_destroy(gpu_); gpu_ = nullptr; }
        SphParams p = gpu_params_;
        p.spacing_r = (float)this->m_TH.spacing_r;
        p.smoothRadius_h = (float)this->m_TH.smoothRadius_h;
        p.dt = (float)this->m_TH.dt;
        for (int i = 0; i < 3; ++i) {
            p.gravity[i] = (float)this->m_TH.gravity_g[i];
            p.spaceMin[i] = (float)this->m_TH.spaceMin[i];
            p.spaceMax[i] = (float)this->m_TH.spaceMax[i];
        }
        p.soundSpeed_cs = (float)this->m_TH.soundSpeed_cs;
        p.nu = (float)this->m_TH.nu;
        p.densityErro_eta = (float)this->m_TH.densityErro_eta;
        int total = 0;
        for (auto& f : this->m_Fluids) {
            total += (int)f.fluidParticles.size();
            if (!f.fluidParticles.empty()) p.particle_d = (float)f.fluidParticles[0].d;
        }
        if (!this->m_Solids.empty()) p.boundary_visc = (float)this->m_Solids[0].viscosity_alpha;
        // solver constants the reference keeps in the solver object
        if constexpr (Solver == SPHGPU_WCSPH) {
            p.wc_gamma = (float)this->m_DensityPower_gamma;  // WcSph.h:34
            // surface tension and adhesion read m_TH.h / r / bt (WcSph.cpp:124-311)
            p.th_h = (float)this->m_TH.h;
            p.th_r = (float)this->m_TH.r;
            p.th_bt = (float)this->m_TH.bt;
        }
        if constexpr (Solver == SPHGPU_PCISPH) {  // PciSph.h:35
            p.pci_min_iter = this->m_minIterations;
            p.pci_max_iter = this->m_maxIterations;
        }
        // IISph reads the particles' kinematic viscosity (SphBase.h:100,181)
        for (auto& f : this->m_Fluids)
            if (!f.fluidParticles.empty()) { p.iv_kvisc = (float)f.fluidParticles[0].kinematicViscosity; break; }
        for (auto& s : this->m_Solids)
            if (!s.boundaryParticles.empty()) { p.iv_kvisc_b = (float)s.boundaryParticles[0].kinematicViscosity; break; }
        int rc = sphgpu_create(&p, device_, total > 0 ? total : 1, &gpu_);
        if (rc) fail("sphgpu_create", rc);
        std::vector<float> xyz, vel;
        std::vector<int> sid;
        for (size_t k = 0; k < this->m_Solids.size(); ++k)
            for (auto& q : this->m_Solids[k].boundaryParticles) {
                for (int c = 0; c < 3; ++c) xyz.push_back((float)q.position[c]);
                sid.push_back((int)k);
            }
        rc = sphgpu_set_boundary(gpu_, (int)sid.size(), xyz.data(), sid.data(), nullptr);
        if (rc) fail("sphgpu_set_boundary", rc);
        counts_.clear();
        for (auto& f : this->m_Fluids) {
            xyz.clear();
            vel.clear();
            for (auto& q : f.fluidParticles)
                for (int c = 0; c < 3; ++c) {
                    xyz.push_back((float)q.position[c]);
                    vel.push_back((float)q.velocity[c]);
                }
            counts_.push_back(f.fluidParticles.size());
            if (f.fluidParticles.empty()) continue;
            rc = sphgpu_add_fluid(gpu_, (int)f.fluidParticles.size(), xyz.data(), vel.data(),
                                  (float)f.restDensity_rho0, (float)f.viscosity_alpha);
            if (rc < 0) fail("sphgpu_add_fluid", rc);
        }
        bool dyn = false;
        for (size_t k = 0; k < this->m_Solids.size(); ++k) {
            auto& s = this->m_Solids[k];
            if (!s.dynamic) continue;
            xyz.clear();
            for (auto& x : s.innerPositions)
                for (int c = 0; c < 3; ++c) xyz.push_back((float)x[c]);
            const SphRigidState st = gpuRigidState((int)k);
            rc = sphgpu_set_solid_dynamic(gpu_, (int)k, xyz.data(), &st);
            if (rc) fail("sphgpu_set_solid_dynamic", rc);
            dyn = true;
        }
        if (dyn) sphgpu_set_rigid_callback(gpu_, &GpuSolver::rigid_trampoline, this);
    }

    // dynamic solids' particles (reference order: solid by solid) back into
    // m_Solids, as updatePaticles leaves them
    void download_solids() {
        bool dyn = false;
        for (auto& s : this->m_Solids) dyn = dyn || s.dynamic;
        if (!dyn) return;
        size_t nb = 0;
        for (auto& s : this->m_Solids) nb += s.boundaryParticles.size();
        std::vector<float> x(3 * nb), v(3 * nb);
        int rc = sphgpu_get_boundary(gpu_, "position", x.data());
        if (rc >= 0) rc = sphgpu_get_boundary(gpu_, "velocity", v.data());
        if (rc < 0) fail("sphgpu_get_boundary", rc);
        size_t i = 0;
        for (auto& s : this->m_Solids) {
            for (auto& q : s.boundaryParticles) {
                if (s.dynamic)
                    for (int c = 0; c < 3; ++c) {
                        q.position[c] = x[3 * i + c];
                        q.velocity[c] = v[3 * i + c];
                    }
                ++i;
            }
        }
    }

    void download() {
        const int n = sphgpu_num_fluid(gpu_);
        if (n < 0) fail("sphgpu_num_fluid", n);
        std::vector<float> xyz(3 * (size_t)n), vel(3 * (size_t)n), rho((size_t)n), ph((size_t)n);
        int rc = sphgpu_get_fluid(gpu_, "position", xyz.data());
        if (rc >= 0) rc = sphgpu_get_fluid(gpu_, "velocity", vel.data());
        if (rc >= 0) rc = sphgpu_get_fluid(gpu_, Solver == SPHGPU_IISPH ? "sphDensity" : "density", rho.data());
        if (rc >= 0) rc = sphgpu_get_fluid(gpu_, "phase", ph.data());
        if (rc < 0) fail("sphgpu_get_fluid", rc);
        // reference order: phase by phase, each in index order; removed
        // particles are gone, so each phase keeps its first survivors
        size_t i = 0;
        for (size_t k = 0; k < this->m_Fluids.size(); ++k) {
            auto& parts = this->m_Fluids[k].fluidParticles;
            size_t m = 0;
            while (i + m < (size_t)n && (size_t)ph[i + m] == k) ++m;
            if (m < parts.size()) parts.resize(m);
            for (size_t j = 0; j < m; ++j) {
                auto& q = parts[j];
                for (int c = 0; c < 3; ++c) {
                    q.position[c] = xyz[3 * (i + j) + c];
                    q.velocity[c] = vel[3 * (i + j) + c];
                }
                if constexpr (Solver == SPHGPU_IISPH) q.sphDensity = rho[i + j];
                else q.density = rho[i + j];
            }
            counts_[k] = parts.size();
            i += m;
        }
    }
};

#endif /* SPHGPU_SOLVER_HPP_ */
