/* Stand-in for the reference's SphWithIO/SphWithBullet layers
 * (SphWithIO.h:25, SphWithBullet.h:40).  The solver classes derive from
 * SphWithIO and call updateSolids() once per step (e.g. DFSPH.cpp:54).
 * Scene construction (addFluidCuboid, addRigidCuboid) is done by the oracle
 * harness filling m_Fluids/m_Solids directly.  Test infrastructure only.
 *
 * updateSolids() follows SphWithBullet::updateSolids
 * (SphWithBullet.cpp:180-224) for dynamic rigid solids, with a host callback
 * in place of the Bullet world: it joins each dynamic solid's boundary forces
 * with the reference's own SphSolid::rigidForceJoin (SphBase.cpp:131-143)
 * about the body's centre of mass, hands force and torque to the callback,
 * which advances the bodies by dt and returns their new states (OpenGL
 * transform, centre of mass, linear and angular velocity, as
 * SphSolid::updatePaticles() reads them from Bullet, SphWithBullet.cpp:
 * 302-317), and moves the boundary particles with the reference's own
 * SphSolid::updatePaticles(com, transform, v, w) (SphBase.cpp:95-128).
 * Static walls are untouched, so with no dynamic solid the call changes
 * nothing.  adjustSpace is not called: the test scenes keep every solid
 * inside the domain. */
#ifndef SPH_WITH_IO_H_
#define SPH_WITH_IO_H_
#include <vector>
#include "SphBase.h"
class SphWithIO : public SphBase {
public:
    /* state: 25 doubles per solid, transform[16] (column-major), com[3],
     * linear[3], angular[3]; returns nonzero on failure */
    typedef int (*RigidFn)(void* user, int nsolids, const int* ids, const double* force, const double* torque,
                           double dt, double* states);
    RigidFn rigid_fn = nullptr;
    void* rigid_user = nullptr;
    int rigid_err = 0;
    struct RigidState {
        float T[16];
        vec_t com, lin;
        vec3_t ang;
    };
    std::vector<RigidState> rigid_state;  // per solid index

    void setRigidState(int k, const double* st) {
        if (int(rigid_state.size()) <= k) rigid_state.resize(k + 1);
        RigidState& r = rigid_state[k];
        for (int c = 0; c < 16; ++c) r.T[c] = float(st[c]);
        for (int c = 0; c < 3; ++c) {
            r.com[c] = real_t(float(st[16 + c]));
            r.lin[c] = real_t(float(st[19 + c]));
            r.ang[c] = real_t(float(st[22 + c]));
        }
    }
    void placeSolid(int k) {
        const RigidState& r = rigid_state[k];
        m_Solids[k].updatePaticles(r.com, r.T, r.lin, r.ang);
    }

protected:
    void updateSolids() {
        std::vector<int> ids;
        std::vector<double> force, torque, states;
        for (int k = 0; k < int(m_Solids.size()); ++k) {
            if (!m_Solids[k].dynamic || k >= int(rigid_state.size())) continue;
            const RigidState& r = rigid_state[k];
            vec_t f;
            vec3_t t;
            m_Solids[k].rigidForceJoin(r.com, f, t);
            ids.push_back(k);
            for (int c = 0; c < 3; ++c) { force.push_back(double(f[c])); torque.push_back(double(t[c])); }
            for (int c = 0; c < 16; ++c) states.push_back(double(r.T[c]));
            for (int c = 0; c < 3; ++c) states.push_back(double(r.com[c]));
            for (int c = 0; c < 3; ++c) states.push_back(double(r.lin[c]));
            for (int c = 0; c < 3; ++c) states.push_back(double(r.ang[c]));
        }
        if (ids.empty()) return;
        if (rigid_fn && rigid_fn(rigid_user, int(ids.size()), ids.data(), force.data(), torque.data(),
                                 double(m_TH.dt), states.data()))
            rigid_err = 1;
        for (size_t j = 0; j < ids.size(); ++j) {
            setRigidState(ids[j], states.data() + 25 * j);
            placeSolid(ids[j]);
        }
    }
};
#endif
