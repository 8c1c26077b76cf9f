// Internal interface of the demag convolution (hsb_demag.cu, hsb_arne.cu).
#pragma once
#include <cuda_runtime.h>

typedef struct hsb_demag_plan_s* hsb_demag_plan;

// Tensor component order of the demag kernel (reference common/index.go:23-28).
enum { KXX = 0, KYY = 1, KZZ = 2, KYZ = 3, KXZ = 4, KXY = 5 };

// Geometry of one Kernel_Arne evaluation (program order, logic size).
struct ArneGeom {
    int size[3];
    long r1[3], r2[3];
    double cs[3];
    double Lmin, accuracy;
    int h[3];  // size/2: the folded octant is [0, h] per axis
};

cudaError_t hsb_arne_launch(const ArneGeom* g, double* Kc, cudaStream_t st);
// The FP64 Newell tensor K = -N in the same folded layout (hsb_newell.cu).
cudaError_t hsb_newell_launch(const ArneGeom* g, double* Kc, cudaStream_t st);
cudaError_t hsb_arne_expand_launch(const double* Kc, int comp, int L0, int L1, int L2, double* out,
                                   cudaStream_t st);

// H (A/m, FP32 SoA [3][N0][N1][N2]) = Ms0 * (K conv (m * mask)); enqueued on st.
// Input/output buffers chosen on the device: m = m[(*msel) ^ minv] (m[0] when msel is
// null), likewise h.  Lets a captured integrator step alternate state buffers without copies.
struct HsbDemagIO {
    const float* m[2];
    const int* msel;
    int minv;
    float* h[2];
    const int* hsel;
    int hinv;
    cudaEvent_t* ev;   // optional: 4 events recorded before x-fwd, after x-fwd, after y/z, after x-inv
};

// Batched convolutions (one per slot, slot = blockIdx.z) on the fast kernels: slot s reads
// m + s * m_stride (its selector msel + s * sel_stride), writes h + s * h_stride, uses the
// spectrum scratch X1 + s * x1_stride (complex elements) and scales by
// scale[s * scale_stride]; `active` is read at active + s * sel_stride.
struct HsbDemagBatch {
    int nslot;
    long m_stride, h_stride;   // floats
    int sel_stride;            // ints
    void* X1;                  // nslot spectra (hsb_demag_x1_bytes each)
    long x1_stride;            // complex elements between slots' spectra
    const float* scale;
    int scale_stride;          // floats
    const float* kern;         // per-slot kernel spectra, fast y/z layout (null: the plan's own)
    long kern_stride;          // floats
};

// `active` (device, nullable): when it points to 0 every kernel returns at once, so a
// captured solver attempt past its target costs only the launches.
int hsb_demag_launch(hsb_demag_plan P, const HsbDemagIO& io, const float* mask, float ms0,
                     cudaStream_t st, const int* active, const HsbDemagBatch* batch = nullptr);
// Bytes of one slot's spectrum scratch; 0 when the plan has no batched (fast) kernels.
long hsb_demag_x1_bytes(hsb_demag_plan P);

// Kernel spectra for other cell sizes on the plan's grid (a batch gives every slot its own,
// exactly as a plan created for that slot's cells would hold).
struct hsb_demag_spec_s;
long hsb_demag_kern_floats(hsb_demag_plan P);
long hsb_demag_spectrum_scratch_bytes(hsb_demag_plan P);
int hsb_demag_spectrum_scratch_create(hsb_demag_plan P, hsb_demag_spec_s** out);
void hsb_demag_spectrum_scratch_destroy(hsb_demag_spec_s* s);
int hsb_demag_spectrum_enqueue(hsb_demag_plan P, const double* cellsize, int accuracy, hsb_demag_spec_s* s,
                               float* kern, float* kern4, cudaStream_t st);
extern "C" int hsb_demag_plan_create(const int* size, const double* cellsize, const int* pbc,
                                     int accuracy, void* stream, hsb_demag_plan* out);
extern "C" int hsb_demag_plan_create_tensor(const int* size, const double* cellsize, const int* pbc, int accuracy,
                                            int tensor, void* stream, hsb_demag_plan* out);
extern "C" int hsb_demag_plan_destroy(hsb_demag_plan P);
// Kernel launches of one convolution (3 fused, 5 multi-pass).
int hsb_demag_nlaunch(hsb_demag_plan P);
