#ifndef CTL_CUDARAYCASTERPROJECTOR_H
#define CTL_CUDARAYCASTERPROJECTOR_H

// CTL AbstractProjector implementation on top of libctlcu.so (include/ctlcu.h).
//
// Drop-in for CTL::OCL::RayCasterProjector (modules/src/projectors/raycasterprojector.h:20-58):
// the same configure()/project() semantics, the same Settings fields and the
// same parameter() keys ("Rays per pixel X/Y", "Ray sampling step length",
// "Volume upsampling factor", "Interpolate", raycasterprojector.cpp:69-91),
// plus the B200 options.  It composes with CTL's ProjectorExtensions exactly
// like the OpenCL projector, because they only call configure() and project().
//
// Builds inside a CTL source tree (needs Qt5 Core and CTL's headers); link
// with -lctlcu.

#include "acquisition/geometryencoder.h"
#include "projectors/abstractprojector.h"

#include "ctlcu.h"

#include <vector>

namespace CTL {
namespace CUDA {

class CudaRayCasterProjector : public AbstractProjector
{
    CTL_TYPE_ID(1001)

public:
    class Settings
    {
    public:
        std::vector<uint> deviceIDs;                //!< CUDA device ordinals (if empty: use all), as
                                                    //!< RayCasterProjector::Settings::deviceIDs
        uint raysPerPixel[2] = { 1, 1 };            //!< sub-rays per pixel along channels (x) and rows (y)
        float raySampling = 0.3f;                   //!< step as a fraction of the smallest voxel size
        uint volumeUpSampling = 1;                  //!< 0: mean voxel, 1: as is, f: f^3 replication
        bool interpolate = true;                    //!< trilinear (true) or nearest voxel (false)
        int interpolationMode = CTLCU_INTERP_SOFTWARE; //!< software FP32 or hardware texture filter
        int accumulation = CTLCU_ACCUM_KAHAN;       //!< FP64, Kahan FP32 or plain FP32
        int storage = CTLCU_F32;                    //!< device storage of the volume (F32, BF16, F16)
        int kernel = CTLCU_KERNEL_AUTO;             //!< sample-loop variant
        uint volumeCacheSize = 4;                   //!< resident copies of recently projected volumes kept
                                                    //!< per device (0: upload every call, as the reference)

        static Settings optimizedFor(const VolumeData& volume, const AbstractDetector& detector);
    };

    CudaRayCasterProjector();
    ~CudaRayCasterProjector() override;

    void configure(const AcquisitionSetup& setup) override;
    ProjectionData project(const VolumeData& volume) override;

    QVariant toVariant() const override;
    QVariant parameter() const override;
    void setParameter(const QVariant& parameter) override;

    Settings& settings();

private:
    ctlcu_settings cSettings() const;

    Settings _settings;
    SingleViewData::Dimensions _viewDim;
    FullGeometry _pMats;
    std::vector<double> _pmatBuffer;  //!< [view][module] row-major 3x4 matrices
    void ensureGroup();

    ctlcu_group* _group = nullptr;    //!< one context per device of _groupIDs
    std::vector<uint> _groupIDs;      //!< deviceIDs the group was made for
};

} // namespace CUDA
} // namespace CTL

#endif // CTL_CUDARAYCASTERPROJECTOR_H
