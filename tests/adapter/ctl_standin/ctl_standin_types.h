// Stand-in for the CTL types that CudaRayCasterProjector uses, with CTL's
// names and the signatures the adapter calls:
//   img/voxelvolume.h (VolumeData = VoxelVolume<float>), img/projectiondata.h,
//   img/singleviewdata.h, acquisition/acquisitionsetup.h, acquisition/ctsystem.h,
//   components/abstractdetector.h, mat/projectionmatrix.h,
//   acquisition/viewgeometry.h (FullGeometry), io/serializationinterface.h.
// The geometry is given directly as projection matrices (the encoder is
// CTL's own and out of scope here).  Test code only.
#ifndef CTL_STANDIN_TYPES_H
#define CTL_STANDIN_TYPES_H

#include "QtStandin.h"

#include <cstddef>
#include <functional>
#include <vector>

using uint = unsigned int;

#define CTL_TYPE_ID(n)
#define DECLARE_SERIALIZABLE_TYPE(T)

namespace CTL {

struct Coord3f { float x, y, z; };
struct Coord3u { uint x, y, z; };

// VoxelVolume<float>: x fastest, index z*X*Y + y*X + x
class VolumeData
{
public:
    VolumeData(Coord3u n, Coord3f voxel, Coord3f offset, std::vector<float> data)
        : _n(n), _voxel(voxel), _offset(offset), _data(std::move(data)) {}
    bool hasData() const { return !_data.empty() && _data.size() == size_t(_n.x) * _n.y * _n.z; }
    float smallestVoxelSize() const { return std::min(std::min(_voxel.x, _voxel.y), _voxel.z); }
    Coord3u nbVoxels() const { return _n; }
    Coord3f voxelSize() const { return _voxel; }
    Coord3f offset() const { return _offset; }
    const float* rawData() const { return _data.data(); }

private:
    Coord3u _n;
    Coord3f _voxel, _offset;
    std::vector<float> _data;
};

class Chunk2D
{
public:
    Chunk2D(uint w, uint h) : _data(size_t(w) * h, 0.0f) {}
    float* rawData() { return _data.data(); }
    const float* rawData() const { return _data.data(); }
    size_t size() const { return _data.size(); }

private:
    std::vector<float> _data;
};

class SingleViewData
{
public:
    struct Dimensions
    {
        uint nbChannels = 0;
        uint nbRows = 0;
        uint nbModules = 0;
    };
    explicit SingleViewData(const Dimensions& d) : _dim(d)
    {
        for(uint m = 0; m < d.nbModules; ++m)
            _modules.emplace_back(d.nbChannels, d.nbRows);
    }
    Chunk2D& module(uint m) { return _modules.at(m); }
    const Chunk2D& module(uint m) const { return _modules.at(m); }
    uint nbModules() const { return uint(_modules.size()); }

private:
    Dimensions _dim;
    std::vector<Chunk2D> _modules;
};

class ProjectionData
{
public:
    explicit ProjectionData(const SingleViewData::Dimensions& d) : _dim(d) {}
    void allocateMemory(uint nbViews)
    {
        _views.clear();
        for(uint v = 0; v < nbViews; ++v)
            _views.emplace_back(_dim);
    }
    uint nbViews() const { return uint(_views.size()); }
    SingleViewData& view(uint v) { return _views.at(v); }
    const SingleViewData& view(uint v) const { return _views.at(v); }
    SingleViewData::Dimensions viewDimensions() const { return _dim; }

private:
    SingleViewData::Dimensions _dim;
    std::vector<SingleViewData> _views;
};

class ProjectionMatrix
{
public:
    double operator()(uint r, uint c) const { return _m[r * 4 + c]; }
    double& operator()(uint r, uint c) { return _m[r * 4 + c]; }

private:
    double _m[12] = {};
};

class SingleViewGeometry
{
public:
    const ProjectionMatrix& at(uint m) const { return _pm.at(m); }
    std::vector<ProjectionMatrix>& modules() { return _pm; }

private:
    std::vector<ProjectionMatrix> _pm;
};

class FullGeometry
{
public:
    uint nbViews() const { return uint(_views.size()); }
    const SingleViewGeometry& at(uint v) const { return _views.at(v); }
    std::vector<SingleViewGeometry>& views() { return _views; }

private:
    std::vector<SingleViewGeometry> _views;
};

class AbstractDetector
{
public:
    AbstractDetector(QSize pixelsPerModule, QSizeF pixelDims, uint modules)
        : _pix(pixelsPerModule), _dims(pixelDims), _modules(modules) {}
    QSize nbPixelPerModule() const { return _pix; }
    QSizeF pixelDimensions() const { return _dims; }
    uint nbDetectorModules() const { return _modules; }

private:
    QSize _pix;
    QSizeF _dims;
    uint _modules;
};

class CTSystem
{
public:
    explicit CTSystem(AbstractDetector d) : _detector(d) {}
    const AbstractDetector* detector() const { return &_detector; }

private:
    AbstractDetector _detector;
};

// AcquisitionSetup: the system and the per-view geometry it encodes to
class AcquisitionSetup
{
public:
    AcquisitionSetup(CTSystem system, FullGeometry geometry) : _system(system), _geometry(geometry) {}
    const CTSystem* system() const { return &_system; }
    const FullGeometry& geometry() const { return _geometry; }
    uint nbViews() const { return _geometry.nbViews(); }

private:
    CTSystem _system;
    FullGeometry _geometry;
};

class SerializationInterface
{
public:
    virtual ~SerializationInterface() = default;
    virtual void fromVariant(const QVariant&) {}
    virtual QVariant toVariant() const { return QVariant(QVariantMap()); }
};

class ProjectorNotifier
{
public:
    std::function<void(int)> onProjectionFinished;
    void projectionFinished(int view)
    {
        if(onProjectionFinished)
            onProjectionFinished(view);
    }
};

} // namespace CTL

#endif
