#include "cudaraycasterprojector.h"
#include "components/abstractdetector.h"

#include <QDebug>
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

namespace CTL {
namespace CUDA {

DECLARE_SERIALIZABLE_TYPE(CudaRayCasterProjector)

// The reference constructor throws std::runtime_error when OpenCL or its
// kernels are missing (raycasterprojector.cpp:388-422); this one throws when
// no CUDA device can be bound.  Like OpenCLConfig, it binds every device of
// the (default, empty = all) device list up front.
CudaRayCasterProjector::CudaRayCasterProjector() { ensureGroup(); }

CudaRayCasterProjector::~CudaRayCasterProjector()
{
    if(_group)
        ctlcu_group_destroy(_group);
}

// One context per listed device, rebuilt when deviceIDs changes; an ordinal
// that does not exist throws, as prepareOpenCLDeviceList does
// (raycasterprojector.cpp:434-461).
void CudaRayCasterProjector::ensureGroup()
{
    if(_group && _groupIDs == _settings.deviceIDs)
        return;
    std::vector<int> ids(_settings.deviceIDs.begin(), _settings.deviceIDs.end());
    ctlcu_group* group = nullptr;
    const int rc = ctlcu_group_create(ids.data(), uint32_t(ids.size()), &group);
    if(rc != CTLCU_OK)
        throw std::runtime_error("CudaRayCasterProjector: device ID is not available or no usable CUDA "
                                 "device (ctlcu status " + std::to_string(rc) + ")");
    if(_group)
        ctlcu_group_destroy(_group);
    _group = group;
    _groupIDs = _settings.deviceIDs;
}

// raycasterprojector.cpp:97-107
void CudaRayCasterProjector::configure(const AcquisitionSetup& setup)
{
    _pMats = GeometryEncoder::encodeFullGeometry(setup);

    auto detectorPixels = setup.system()->detector()->nbPixelPerModule();
    _viewDim.nbRows = uint(detectorPixels.height());
    _viewDim.nbChannels = uint(detectorPixels.width());
    _viewDim.nbModules = setup.system()->detector()->nbDetectorModules();

    // FullGeometry -> [view][module] row-major 3x4 doubles (the C ABI's input)
    const uint nbViews = _pMats.nbViews();
    _pmatBuffer.assign(size_t(nbViews) * _viewDim.nbModules * 12, 0.0);
    auto* p = _pmatBuffer.data();
    for(uint v = 0; v < nbViews; ++v)
        for(uint m = 0; m < _viewDim.nbModules; ++m)
        {
            const auto& P = _pMats.at(v).at(m);
            for(uint r = 0; r < 3; ++r)
                for(uint c = 0; c < 4; ++c)
                    *p++ = P(r, c);
        }
}

ctlcu_settings CudaRayCasterProjector::cSettings() const
{
    ctlcu_settings s = ctlcu_settings_default();
    s.rays_per_pixel[0] = _settings.raysPerPixel[0];
    s.rays_per_pixel[1] = _settings.raysPerPixel[1];
    s.ray_sampling = _settings.raySampling;
    s.volume_upsampling = _settings.interpolate ? _settings.volumeUpSampling : 1u;
    s.interpolate = _settings.interpolate ? 1 : 0;
    s.interp_mode = _settings.interpolationMode;
    s.accum = _settings.accumulation;
    s.kernel = _settings.kernel;
    return s;
}

// raycasterprojector.cpp:139-375 with the same error behaviour: an invalid
// volume returns empty ProjectionData, a device error returns the (zero) result
ProjectionData CudaRayCasterProjector::project(const VolumeData& volume)
{
    if(!_settings.interpolate)
        _settings.volumeUpSampling = 1;

    ProjectionData ret(_viewDim);
    if(!volume.hasData())
    {
        qCritical() << "no or contradictory data in volume object";
        return ret;
    }
    if(volume.smallestVoxelSize() <= 0.0f)
        qWarning() << "voxel size is zero or negative";

    const uint nbViews = _pMats.nbViews();
    if(nbViews == 0)
    {
        qCritical() << "CudaRayCasterProjector::project: no views configured";
        return ret;
    }
    ensureGroup();
    // repeated projections of one volume (extensions re-projecting it per
    // focal-spot sample or energy bin, a registration loop per pose) reuse the
    // device copy instead of uploading it again; results are the same
    uint32_t nbDevices = 0;
    ctlcu_group_size(_group, &nbDevices);
    for(uint32_t i = 0; i < nbDevices; ++i)
    {
        ctlcu_ctx* ctx = nullptr;
        if(ctlcu_group_context(_group, i, &ctx) == CTLCU_OK)
            ctlcu_set_volume_cache(ctx, _settings.volumeCacheSize);
    }

    ctlcu_volume_desc desc;
    desc.n[0] = volume.nbVoxels().x;
    desc.n[1] = volume.nbVoxels().y;
    desc.n[2] = volume.nbVoxels().z;
    desc.voxel_mm[0] = volume.voxelSize().x;
    desc.voxel_mm[1] = volume.voxelSize().y;
    desc.voxel_mm[2] = volume.voxelSize().z;
    desc.offset_mm[0] = volume.offset().x;
    desc.offset_mm[1] = volume.offset().y;
    desc.offset_mm[2] = volume.offset().z;
    desc.dtype = _settings.storage;

    const size_t pixelsPerModule = size_t(_viewDim.nbRows) * _viewDim.nbChannels;
    std::vector<float> out(size_t(nbViews) * _viewDim.nbModules * pixelsPerModule, 0.0f);
    const ctlcu_settings s = cSettings();
    // views in contiguous blocks over the listed devices (raycasterprojector.cpp:321-357
    // deals them out round-robin); one device runs the call on the caller's thread
    const int rc = ctlcu_group_project_volume(_group, &desc, volume.rawData(), &s, _pmatBuffer.data(), nbViews,
                                              _viewDim.nbModules, _viewDim.nbChannels, _viewDim.nbRows,
                                              out.data());
    if(rc != CTLCU_OK && rc != CTLCU_ERR_SINGULAR_GEOMETRY)
        qCritical() << "ctlcu error" << rc << ":" << ctlcu_group_last_error(_group);
    else if(rc == CTLCU_ERR_SINGULAR_GEOMETRY)
        qWarning() << "QR decomposition: matrix is close to singular;" << ctlcu_group_last_error(_group);

    ret.allocateMemory(nbViews);
    const float* src = out.data();
    for(uint v = 0; v < nbViews; ++v)
    {
        for(uint m = 0; m < _viewDim.nbModules; ++m)
        {
            std::copy_n(src, pixelsPerModule, ret.view(v).module(m).rawData());
            src += pixelsPerModule;
        }
        emit notifier()->projectionFinished(int(v));
    }
    return ret;
}

// raycasterprojector.cpp:60-91 (same keys, plus the B200 options)
QVariant CudaRayCasterProjector::toVariant() const
{
    QVariantMap ret = AbstractProjector::toVariant().toMap();
    ret.insert("#", "CudaRayCasterProjector");
    return ret;
}

QVariant CudaRayCasterProjector::parameter() const
{
    QVariantMap ret = AbstractProjector::parameter().toMap();
    ret.insert("Rays per pixel X", _settings.raysPerPixel[0]);
    ret.insert("Rays per pixel Y", _settings.raysPerPixel[1]);
    ret.insert("Ray sampling step length", _settings.raySampling);
    ret.insert("Volume upsampling factor", _settings.volumeUpSampling);
    ret.insert("Interpolate", _settings.interpolate);
    ret.insert("Interpolation mode", _settings.interpolationMode);
    ret.insert("Accumulation", _settings.accumulation);
    ret.insert("Storage", _settings.storage);
    ret.insert("Kernel", _settings.kernel);
    return ret;
}

void CudaRayCasterProjector::setParameter(const QVariant& parameter)
{
    const QVariantMap map = parameter.toMap();
    _settings.raysPerPixel[0] = map.value("Rays per pixel X", 1u).toUInt();
    _settings.raysPerPixel[1] = map.value("Rays per pixel Y", 1u).toUInt();
    _settings.raySampling = map.value("Ray sampling step length", 0.3f).toFloat();
    _settings.volumeUpSampling = map.value("Volume upsampling factor", 1u).toUInt();
    _settings.interpolate = map.value("Interpolate", true).toBool();
    _settings.interpolationMode = map.value("Interpolation mode", int(CTLCU_INTERP_SOFTWARE)).toInt();
    _settings.accumulation = map.value("Accumulation", int(CTLCU_ACCUM_KAHAN)).toInt();
    _settings.storage = map.value("Storage", int(CTLCU_F32)).toInt();
    _settings.kernel = map.value("Kernel", int(CTLCU_KERNEL_AUTO)).toInt();
}

CudaRayCasterProjector::Settings& CudaRayCasterProjector::settings() { return _settings; }

// raycasterprojector.cpp:482-521
CudaRayCasterProjector::Settings
CudaRayCasterProjector::Settings::optimizedFor(const VolumeData& volume, const AbstractDetector& detector)
{
    Settings ret;
    const double Xmm = detector.pixelDimensions().width();
    const double Ymm = detector.pixelDimensions().height();
    if(Xmm == 0.0 || Ymm == 0.0)
        throw std::runtime_error("pixel dimensions are singular");
    double pixelRatio = Xmm / Ymm;
    const bool broadPixel = pixelRatio > 1.0;
    if(broadPixel)
        pixelRatio = 1.0 / pixelRatio;
    const uint ratios[5][2] = { { 1, 2 }, { 1, 3 }, { 1, 4 }, { 2, 3 }, { 3, 4 } };
    double deviation = std::fabs(pixelRatio - 1.0);
    for(const auto& r : ratios)
        if(std::fabs(pixelRatio - double(r[0]) / double(r[1])) < deviation)
        {
            deviation = std::fabs(pixelRatio - double(r[0]) / double(r[1]));
            ret.raysPerPixel[0] = r[broadPixel];
            ret.raysPerPixel[1] = r[!broadPixel];
        }
    const auto smallestVoxelSize = double(volume.smallestVoxelSize());
    const auto smallestPixelSize = std::min(Xmm / ret.raysPerPixel[0], Ymm / ret.raysPerPixel[1]);
    ret.volumeUpSampling = std::max(uint(smallestVoxelSize / smallestPixelSize), 1u);
    const uint rayIncreaseFactor = std::max(uint(smallestPixelSize / smallestVoxelSize), 1u);
    ret.raysPerPixel[0] *= rayIncreaseFactor;
    ret.raysPerPixel[1] *= rayIncreaseFactor;
    return ret;
}

} // namespace CUDA
} // namespace CTL
