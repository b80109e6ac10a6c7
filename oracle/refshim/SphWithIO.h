/* Stand-in for the reference's SphWithIO/SphWithBullet layers
 * (SphWithIO.h:25, SphWithBullet.h:40).  The solver classes derive from
 * SphWithIO and call updateSolids() once per step (e.g. DFSPH.cpp:54); with
 * static walls that call changes nothing, so the stand-in is a no-op.  Scene
 * construction (addFluidCuboid, addRigidCuboid) is done by the oracle harness
 * filling m_Fluids/m_Solids directly.  Test infrastructure only. */
#ifndef SPH_WITH_IO_H_
#define SPH_WITH_IO_H_
#include "SphBase.h"
class SphWithIO : public SphBase {
protected:
    void updateSolids() {}
};
#endif
