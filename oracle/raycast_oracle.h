/*
 * FP64 CPU oracle for the cone-beam forward projector -- TEST INFRASTRUCTURE.
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg, always as the checker, never as the product path.
 */
#ifndef CTLB200_RAYCAST_ORACLE_H
#define CTLB200_RAYCAST_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_OK = 0, ORACLE_ERR_ARG = 1, ORACLE_ERR_ALLOC = 2 };

typedef struct {
    long long n[3];      /* voxels along x, y, z (x fastest in memory) */
    float voxel_mm[3];   /* voxel size */
    float offset_mm[3];  /* volume centre */
} oracle_volume;

typedef struct {
    unsigned rays_per_pixel[2]; /* sub-rays along channel (x) and row (y) */
    float ray_sampling;         /* step as a fraction of the smallest voxel size */
    unsigned volume_upsampling; /* 0: one mean voxel, 1: unchanged, f>=2: f^3 replication */
    int interpolate;            /* 1: trilinear, 0: nearest voxel (forces up-sampling 1) */
} oracle_settings;

/* pmats: n_views * n_modules row-major 3x4 matrices; out: [view][module][row][channel]. */
int oracle_project(const float* volume, const oracle_volume* vd, const oracle_settings* s,
                   const double* pmats, unsigned n_views, unsigned n_modules,
                   unsigned channels, unsigned rows, float* out,
                   unsigned long long* sample_count, int n_threads);

void oracle_source_position(const double P[12], double src[3]);
int oracle_decompose_m(const double M[9], double qr[15]);
int oracle_view_setup(const double* pmats, unsigned n_views, unsigned n_modules,
                      double* qr_out, double* src_out);

#ifdef __cplusplus
}
#endif
#endif
