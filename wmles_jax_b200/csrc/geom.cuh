// Block geometry and packed metric table on the device (geom.cu).
#pragma once
#include <cuda_runtime.h>

namespace wm {

struct GeomArgs {
    const double* X;             // 3 x (N0+1) x (N1+1) x (N2+1) nodes, ghost nodes filled
    int N[3];                    // cells per direction including ghosts
    double* vol;                 // N0 x N1 x N2
    double* xc;                  // 3 x N0 x N1 x N2
    double* S[3];                // 3 x (N0 + (d==0)) x (N1 + (d==1)) x (N2 + (d==2))
    double* xf[3];               // same extents as S[d]
    double* met;                 // WM_NMET x N0 x N1 x N2, or null
};

cudaError_t launch_geometry(const GeomArgs& A, cudaStream_t s);

// dst[i] = (float)src[i] (round to nearest), i < n
cudaError_t launch_to_f32(const double* src, float* dst, long long n, cudaStream_t s);

}  // namespace wm
