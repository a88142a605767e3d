// ensemble.cuh -- batched ensembles: many independent domains (members) of
// uneven sizes advanced together, every kernel of a time step launched once
// for all members and the step captured in a CUDA graph.
#pragma once

#include "how_internal.cuh"

namespace how {

constexpr int kEnsShapes = 3;   // tile-shape candidates per sweep direction

// shapes, tiles and launches of the batched sweep (ensemble_sweep.cu)
void ens_shape(int dir, int s, int* nl, int* t);
long long ens_tiles(const Grid& g, int dir, int s);
int ens_encode_maps(const Ctx& c, int dir, int s, CUtensorMap* tm_in, CUtensorMap* tm_out);
void ens_launch_sweep(int dir, int s, const SweepArgs& a0, cudaStream_t st, int dev);

// Per-member description read by the batched kernels.  Stage s of q lives in
// qbuf[s], except that stages 0 and 5 trade buffers when par (the member's
// step parity) is 1; face B likewise.
struct EnsMember {
    Grid g;
    double* qbuf[6];
    double* bbuf[6];
    double* ct[12];
    DevScalars* dsc;
    double gam, rhomin, pgmin, cour, dx, dy, dz, dtout;
    int nt;
    int periodic[3];
    int use_x, use_y, use_z, use_Ox, use_Oy, use_Oz, any_ct;
};

// Per-member time state, advanced on the device.
struct EnsState {
    double time;
    long long steps;
    int out_step;   // output interval being integrated (1..nt)
    int done;       // reached tend (or failed)
    int err;        // 1: non-positive dt
    int pad;
};

}  // namespace how
