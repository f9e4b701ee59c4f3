// Structures shared by the render server's host loop (server.cpp) and its
// device step (k_serve.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device_types.h"

namespace prr {

// One admitted request as the device sees it during a step.
struct ServeReq {
    const DevScene *scene;   // the scene's resident descriptor (device memory)
    DevCamera camera;        // the scene's camera at the request's resolution
    int x0, y0, ww, wh;      // pixel window
    int s0, s1;              // samples of this step's chunk
    int max_depth;
    float clamp;
    uint64_t seed;
    float3 *film;            // ww*wh running sums, zeroed at admission
    unsigned long long rays; // rays traced (closest + shadow)
};

// One block of a step: a 16x8 tile of one request.
struct ServeItem {
    int req;
    int tile;
};

int serve_launch_step(const ServeItem *d_items, int n_items, ServeReq *d_reqs, int tlas_cap,
                      int blas_cap, cudaStream_t st);
int serve_resolve(const float3 *film, int npix, int n, float *out, cudaStream_t st);
int serve_tiles(int ww, int wh);

} // namespace prr
