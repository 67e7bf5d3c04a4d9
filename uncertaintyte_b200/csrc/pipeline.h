// pipeline.h - the stages of computeCovariances shared by the single-scene
// entry points (api.cu) and the grouped batch (batch.cu).
#pragma once
#include "internal.h"

namespace unc {

struct Plan {
    int C, P, nobs, N, ld;
    bool svd_schur;  // UNC_SVD_SCHUR: pseudo-inverse of the camera Schur complement
};

struct Buffers {
    int *rows, *cols;
    double* vals;
    double *cam_out, *pt_out;
    SceneDev s;
    double *Z, *iZ, *add, *tmp, *e, *gjws, *sig;
    double *p4, *p8, *p12, *p16, *g;   // blocked-power Taylor evaluation: X^4, X^8, X^12, X^16, G_q
    unsigned long long* dmax;          // 24 words: the powers' diagonal maxima
    int* dag_state;  // counters of the tile-task inverse
    unsigned long long* amax;
    TeState* te;
    PinvBuffers pb;  // UNC_SVD_SCHUR only
};

Plan make_plan(const unc_options* o, int num_rows);
// Lay out the workspace; with base == nullptr only the size is computed.
// host_io: the input copies (rows, cols, values) and outputs are carved too.
size_t carve(char* base, const Plan& pl, bool host_io, long long nnz, int nrows, Buffers& b);
int check_options(const unc_options* o, int num_rows, int num_cols);
bool is_svd(const unc_options* o);
// Grow-only device buffer allocated in stream order on sm.
int grow_buffer(void** p, size_t* have, size_t need, size_t want, cudaStream_t sm);

// The sparse stages of computeCovariances on stream sm (compute.cpp:73-118,
// 283-368): observation validation (fixPts), the observation index, J^T J
// blocks and column norms, point blocks and their inverses, W/Y, and the
// scaled Schur complement Z = U - W V^-1 W^T (both triangles). No host round
// trip: the stage can be captured in a graph.
// fx receives the fixed points as the reference orders them. ev: 6 events
// recorded at the stage boundaries, or nullptr.
int sparse_stage(const unc_options* o, const Plan& pl, long long nnz, const int* rows, const int* cols,
                 const double* vals, Buffers& b, int fx[3], cudaEvent_t* ev, cudaStream_t sm);

// The camera outputs (removeScaleJ4Z, compute.cpp:168-183) from iZ and the
// point covariances (compute.cpp:370-455, 517-527) into cam_out / pt_out.
void output_stage(const Plan& pl, Buffers& b, double* cam_out, double* pt_out, cudaStream_t sm);

// The automatic lambda of teInverse (compute.cpp:124-125) for N camera parameters.
double auto_lambda(int N);
// factorial() of compute.cpp:57-62: 32-bit signed, wraps from 13! on.
int32_t factorial_i32(int n);

}  // namespace unc
