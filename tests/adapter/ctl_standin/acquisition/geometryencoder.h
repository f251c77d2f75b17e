// Stand-in for CTL's acquisition/geometryencoder.h: the setup already holds
// its projection matrices.  Test code only.
#ifndef CTL_STANDIN_GEOMETRYENCODER_H
#define CTL_STANDIN_GEOMETRYENCODER_H

#include "../ctl_standin_types.h"

namespace CTL {

struct GeometryEncoder
{
    static FullGeometry encodeFullGeometry(const AcquisitionSetup& setup) { return setup.geometry(); }
};

} // namespace CTL

#endif
