/* Drop-in check (test infrastructure, built by oracle/build_ref.py into
 * oracle/_ref/dropin_<solver>): a scene class derived from the reference's
 * own solver class, switched to the GPU by changing its base class to
 * GpuSolver<REF_SOLVER_CLASS, ...> (include/sphgpu_solver.hpp).  The scene
 * is read from a binary file, advanced with the reference's runOneStep()
 * (SphBase.cpp:348-354), and the particles of m_Fluids are written back out:
 *
 *   dropin_<solver> in.bin out.bin
 *
 * in.bin:  int32 nf, nb, steps; float32 spacing_r, smoothRadius_h, dt,
 *          gravity[3], spaceMin[3], spaceMax[3], soundSpeed_cs, nu, rho0,
 *          visc_alpha, boundary_visc, d, density_goal, div_goal_rel,
 *          densityErro_eta;
 *          then fluid positions[nf*3], velocities[nf*3], boundary positions[nb*3];
 *          optionally int32 nbody and, if nbody > 0, a dynamic rigid solid
 *          (solid 1): float32 body-frame positions[nbody*3], centre of mass
 *          at t = 0 [3], linear velocity [3], angular velocity about z --
 *          a body in prescribed motion (translation plus rotation about z
 *          through the centre of mass), which gpuRigidStep advances
 * out.bin: int32 n, frame, total density iterations; float32 positions[n*3],
 *          velocities[n*3], densities[n] (m_Fluids[0] after the steps;
 *          IISph: sphDensity); with a body also float32 its particles'
 *          positions[nbody*3] and the force and torque (float64[6]) of the
 *          last step */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include REF_SOLVER_HEADER
#include "sphgpu_solver.hpp"

class DropinScene : public GpuSolver<REF_SOLVER_CLASS, REF_SPHGPU_SOLVER> {
public:
    void setupScene() override {}
    void stepEvent() override {}

    int iters = 0;
    // prescribed motion of the dynamic body (solid 1)
    int nbody = 0;
    float com0[3] = {0, 0, 0}, lin[3] = {0, 0, 0}, wz = 0;
    double t = 0;
    double last_ft[6] = {0, 0, 0, 0, 0, 0};

    SphRigidState body_state(double time) const {
        SphRigidState s = {};
        const double a = (double)wz * time, c = std::cos(a), sn = std::sin(a);
        s.transform[0] = (float)c;
        s.transform[1] = (float)sn;
        s.transform[4] = (float)-sn;
        s.transform[5] = (float)c;
        s.transform[10] = 1.f;
        s.transform[15] = 1.f;
        for (int k = 0; k < 3; ++k) {
            const float x = (float)((double)com0[k] + (double)lin[k] * time);
            s.transform[12 + k] = x;
            s.center_of_mass[k] = x;
            s.linear_velocity[k] = lin[k];
        }
        s.angular_velocity[2] = wz;
        return s;
    }
    SphRigidState gpuRigidState(int) override { return body_state(t); }
    void gpuRigidStep(int n, const int*, const double* force, const double* torque, double dt,
                      SphRigidState* states) override {
        for (int k = 0; k < 3; ++k) { last_ft[k] = force[k]; last_ft[3 + k] = torque[k]; }
        t += dt;
        for (int i = 0; i < n; ++i) states[i] = body_state(t);
    }

    void load(FILE* f, int& steps) {
        int32_t hdr[3];
        float q[24];
        if (fread(hdr, sizeof hdr, 1, f) != 1 || fread(q, sizeof q, 1, f) != 1) exit(2);
        const int nf = hdr[0], nb = hdr[1];
        steps = hdr[2];
        m_TH.spacing_r = q[0];
        m_TH.smoothRadius_h = q[1];
        m_TH.dt = q[2];
        m_TH.gravity_g = vec_t(q[3], q[4], q[5]);
        m_TH.spaceMin = vec_t(q[6], q[7], q[8]);
        m_TH.spaceMax = vec_t(q[9], q[10], q[11]);
        m_TH.soundSpeed_cs = q[12];
        m_TH.nu = q[13];
        m_TH.densityErro_eta = q[20];  // PciSph's loop goal (uninitialised in ThresholdsBase)
        m_TH.h = q[21];  // WcSph's surface tension and adhesion (uninitialised in ThresholdsBase)
        m_TH.r = q[22];
        m_TH.bt = q[23];
        const float rho0 = q[14], visc = q[15], bvisc = q[16], d = q[17];
        gpuParams().df_density_goal = q[18];
        gpuParams().df_div_goal_abs = 0.0;
        gpuParams().df_div_goal_rel = q[19];
        gpuParams().df_div_max_iter = 100;
        std::vector<float> fp(3 * (size_t)nf), fv(3 * (size_t)nf), bp(3 * (size_t)nb);
        if (fread(fp.data(), sizeof(float), fp.size(), f) != fp.size() ||
            fread(fv.data(), sizeof(float), fv.size(), f) != fv.size() ||
            fread(bp.data(), sizeof(float), bp.size(), f) != bp.size())
            exit(2);
        SphSolid s(false, SphSolid::RIGIDBODY, static_cast<real_t>(bvisc), 0);
        BoundaryParticle b = BoundaryParticle();
        b.d = d;
        b.restDensity = rho0;
        for (int i = 0; i < nb; ++i) {
            b.position = vec_t(bp[3 * i], bp[3 * i + 1], bp[3 * i + 2]);
            s.boundaryParticles.push_back(b);
            s.innerPositions.push_back(b.position);
        }
        m_Solids.push_back(s);
        int32_t nbd = 0;
        if (fread(&nbd, sizeof nbd, 1, f) == 1 && nbd > 0) {
            nbody = nbd;
            std::vector<float> in(3 * (size_t)nbd);
            float m[7];
            if (fread(in.data(), sizeof(float), in.size(), f) != in.size() || fread(m, sizeof m, 1, f) != 1) exit(2);
            for (int k = 0; k < 3; ++k) { com0[k] = m[k]; lin[k] = m[3 + k]; }
            wz = m[6];
            SphSolid body(true, SphSolid::RIGIDBODY, static_cast<real_t>(bvisc), 0);
            for (int i = 0; i < nbd; ++i) {
                const vec_t x0(in[3 * i], in[3 * i + 1], in[3 * i + 2]);
                b.position = vec_t(x0[0] + com0[0], x0[1] + com0[1], x0[2] + com0[2]);
                body.boundaryParticles.push_back(b);
                body.innerPositions.push_back(x0);
            }
            m_Solids.push_back(body);
        }
        SphFluid fl(static_cast<real_t>(rho0), static_cast<real_t>(visc), static_cast<real_t>(0));
        FluidParticle p = FluidParticle();
        p.d = d;
        p.restDensity = rho0;
        p.density = rho0;
        for (int i = 0; i < nf; ++i) {
            p.position = vec_t(fp[3 * i], fp[3 * i + 1], fp[3 * i + 2]);
            p.velocity = vec_t(fv[3 * i], fv[3 * i + 1], fv[3 * i + 2]);
            fl.fluidParticles.push_back(p);
        }
        m_Fluids.push_back(fl);
    }

    void save(FILE* f) {
        const auto& parts = m_Fluids[0].fluidParticles;
        int32_t hdr[3] = {(int32_t)parts.size(), (int32_t)m_TH.frameNumber, iters};
        fwrite(hdr, sizeof hdr, 1, f);
        std::vector<float> x, v, r;
        for (auto& q : parts) {
            for (int c = 0; c < 3; ++c) { x.push_back((float)q.position[c]); v.push_back((float)q.velocity[c]); }
#if REF_SPHGPU_SOLVER == SPHGPU_IISPH
            r.push_back((float)q.sphDensity);
#else
            r.push_back((float)q.density);
#endif
        }
        fwrite(x.data(), sizeof(float), x.size(), f);
        fwrite(v.data(), sizeof(float), v.size(), f);
        fwrite(r.data(), sizeof(float), r.size(), f);
        if (nbody > 0) {
            std::vector<float> bx;
            for (auto& q : m_Solids[1].boundaryParticles)
                for (int c = 0; c < 3; ++c) bx.push_back((float)q.position[c]);
            fwrite(bx.data(), sizeof(float), bx.size(), f);
            fwrite(last_ft, sizeof last_ft, 1, f);
        }
    }
};

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 1;
    }
    FILE* in = fopen(argv[1], "rb");
    if (!in) return 1;
    DropinScene scene;
    int steps = 0;
    scene.load(in, steps);
    fclose(in);
    scene.setupScene();
    try {
        for (int i = 0; i < steps; ++i) {
            scene.runOneStep();
            scene.iters += scene.gpuStats().iter_density;
        }
    } catch (const std::exception& e) {
        fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    FILE* out = fopen(argv[2], "wb");
    if (!out) return 1;
    scene.save(out);
    fclose(out);
    return 0;
}
