// Drives CTL::CUDA::CudaRayCasterProjector (ctl_b200/adapter/) through CTL's
// AbstractProjector interface, compiled against the CTL stand-in headers:
//   adapter_main <dir>
// reads <dir>/meta.txt ("nx ny nz vx vy vz ox oy oz channels rows modules views
// rays_x rays_y ray_sampling upsampling interpolate"), volume.bin (float32,
// x fastest) and pmats.bin (float64 [view][module] 3x4 row-major), then
// configure()s, project()s and writes out.bin (float32 [view][module][row][channel]).
// It also checks that parameter() round-trips through setParameter(), that
// projectionFinished() fires once per view, and that the device lists {0, 0}
// and {0, 0, 0} give the same bits.  Test code only.
#include "cudaraycasterprojector.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

using namespace CTL;

template <typename T>
static std::vector<T> readAll(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<T> out(bytes.size() / sizeof(T));
    std::memcpy(out.data(), bytes.data(), out.size() * sizeof(T));
    return out;
}

int main(int argc, char** argv)
{
    if(argc < 2)
        return 2;
    const std::string dir = argv[1];
    std::ifstream meta(dir + "/meta.txt");
    uint nx, ny, nz, C, R, M, V, rx, ry, up, interp;
    float vx, vy, vz, ox, oy, oz, rs;
    meta >> nx >> ny >> nz >> vx >> vy >> vz >> ox >> oy >> oz >> C >> R >> M >> V >> rx >> ry >> rs >> up >> interp;
    if(!meta)
        return 3;

    VolumeData volume({ nx, ny, nz }, { vx, vy, vz }, { ox, oy, oz }, readAll<float>(dir + "/volume.bin"));
    const auto pm = readAll<double>(dir + "/pmats.bin");
    if(pm.size() != size_t(V) * M * 12)
        return 4;
    FullGeometry geo;
    for(uint v = 0; v < V; ++v)
    {
        SingleViewGeometry g;
        for(uint m = 0; m < M; ++m)
        {
            ProjectionMatrix P;
            for(uint k = 0; k < 12; ++k)
                P(k / 4, k % 4) = pm[(size_t(v) * M + m) * 12 + k];
            g.modules().push_back(P);
        }
        geo.views().push_back(g);
    }
    AcquisitionSetup setup(CTSystem(AbstractDetector(QSize(int(C), int(R)), QSizeF(1.0, 1.0), M)), geo);

    CUDA::CudaRayCasterProjector projector;
    auto& s = projector.settings();
    s.raysPerPixel[0] = rx;
    s.raysPerPixel[1] = ry;
    s.raySampling = rs;
    s.volumeUpSampling = up;
    s.interpolate = interp != 0;

    // parameter() -> setParameter() keeps every setting
    const QVariant params = projector.parameter();
    projector.setParameter(params);
    if(s.raysPerPixel[0] != rx || s.raysPerPixel[1] != ry || s.raySampling != rs ||
       s.volumeUpSampling != up || s.interpolate != (interp != 0))
    {
        std::fprintf(stderr, "parameter round trip changed the settings\n");
        return 5;
    }

    int finished = 0;
    projector.notifier()->onProjectionFinished = [&finished](int) { ++finished; };
    projector.configure(setup);
    const ProjectionData proj = projector.project(volume);
    if(proj.nbViews() != V || finished != int(V))
    {
        std::fprintf(stderr, "views %u, notifications %d, expected %u\n", proj.nbViews(), finished, V);
        return 6;
    }
    std::ofstream out(dir + "/out.bin", std::ios::binary);
    for(uint v = 0; v < V; ++v)
        for(uint m = 0; m < M; ++m)
            out.write(reinterpret_cast<const char*>(proj.view(v).module(m).rawData()),
                      std::streamsize(sizeof(float) * size_t(C) * R));

    // the same projection spread over the device list {0, 0} and {0, 0, 0}
    // (several contexts on one GPU, each with its contiguous block of views):
    // identical bits to the one-device call
    for(uint copies : { 2u, 3u })
    {
        s.deviceIDs.assign(copies, 0u);
        const ProjectionData multi = projector.project(volume);
        if(multi.nbViews() != V)
            return 8;
        for(uint v = 0; v < V; ++v)
            for(uint m = 0; m < M; ++m)
                if(std::memcmp(multi.view(v).module(m).rawData(), proj.view(v).module(m).rawData(),
                               sizeof(float) * size_t(C) * R) != 0)
                {
                    std::fprintf(stderr, "deviceIDs of %u entries: view %u module %u differs\n", copies, v, m);
                    return 9;
                }
    }
    s.deviceIDs.clear();

    // an empty volume gives empty projections and no exception, as in the reference
    VolumeData empty({ 0, 0, 0 }, { 1, 1, 1 }, { 0, 0, 0 }, {});
    if(projector.project(empty).nbViews() != 0)
        return 7;
    return 0;
}
