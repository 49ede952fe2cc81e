// Allocation-free variant of the right-hand-side evaluation.
//
// dndsb_eval_evaluate_rhs keeps its per-face flux scratch in memory the
// evaluator handle allocated with cudaMalloc.  Some host programs must not
// allocate device memory at the point where they evaluate residuals: for
// example an application whose GPU memory is owned entirely by its own pool
// allocator (a raw cudaMalloc would bypass its accounting and fragment the
// pool), or a latency-critical loop that cannot afford the device-wide
// synchronisation cudaMalloc and cudaFree may imply.  For them this file
// keeps the scratch in a fixed-size array of static device memory that every
// GPU loading the library holds until the process exits.
//
// Rules of use:
//  * capacity: nFace * nVars <= DNDSB_NOALLOC_SCRATCH_DOUBLES (2^20 doubles,
//    8 MiB); larger meshes are rejected with DNDSB_E_UNSUPPORTED;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current); make that first call
//    before any stream capture begins;
//  * like dndsb_eval_evaluate_rhs, a call reads the device error word back and
//    synchronises its stream before it returns, unless the evaluator reports
//    its errors deferred (dndsb_eval_set_deferred_errors);
//  * every call on a device shares the one array and leaves the last call's
//    face fluxes in it; no entry has to start at zero because the face kernel
//    writes every entry the gather kernel reads;
//  * calls whose kernels overlap on the GPU (concurrent streams, threads or
//    evaluators on the same device) race on the array; serialise them.
#include "../../include/dndsb.h"
#include "solver.cuh"

#include <mutex>
#include <string>

struct dndsb_mesh;
struct dndsb_vr;
struct dndsb_eval;

namespace dndsb
{
// accessors of the handle internals, defined in capi.cu
const MeshD &mesh_of(const dndsb_eval *e);
const GeomD &geom_of(const dndsb_eval *e);
const VRD &vr_of(const dndsb_eval *e);
bool vr_ready(const dndsb_eval *e);
EvalD &eval_of(dndsb_eval *e);
int set_error(int code, const std::string &msg);
} // namespace dndsb

static __device__ __align__(256) double g_noalloc_face_flux[DNDSB_NOALLOC_SCRATCH_DOUBLES];

namespace
{
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

// once per device, with that device current: the device address of the static array
int scratch_for_current_device(double **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return dndsb::set_error(DNDSB_E_CUDA, "dndsb_eval_evaluate_rhs_noalloc: no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev])
    {
        void *p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_face_flux);
        if (rc != cudaSuccess || !p)
            return dndsb::set_error(DNDSB_E_CUDA, std::string("dndsb_eval_evaluate_rhs_noalloc: cudaGetSymbolAddress failed: ") +
                                                      cudaGetErrorString(rc));
        g_scratch_addr[dev] = (double *)p;
    }
    *out = g_scratch_addr[dev];
    return DNDSB_OK;
}
} // namespace

extern "C" int dndsb_eval_evaluate_rhs_noalloc(dndsb_eval *ev, double *rhs, const double *u, const double *uRec, void *stream)
{
    using namespace dndsb;
    if (!ev || !rhs || !u || !uRec)
        return set_error(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_noalloc: null argument");
    if (!vr_ready(ev))
        return set_error(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_noalloc: VR not constructed");
    const MeshD &m = mesh_of(ev);
    EvalD &e = eval_of(ev);
    if (m.nBndFace > 0 && vr_of(ev).bnd.nZone == 0)
        return set_error(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_noalloc: the mesh has boundary faces; call dndsb_eval_set_bc first");
    int64_t need = m.nFace * (int64_t)e.s.nVars;
    if (need > (int64_t)DNDSB_NOALLOC_SCRATCH_DOUBLES)
        return set_error(DNDSB_E_UNSUPPORTED, "dndsb_eval_evaluate_rhs_noalloc: nFace * nVars = " + std::to_string(need) +
                                                  " exceeds the static scratch of " + std::to_string(DNDSB_NOALLOC_SCRATCH_DOUBLES) +
                                                  " doubles; use dndsb_eval_evaluate_rhs");
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != DNDSB_OK)
        return rc;
    rc = eval_rhs(m, geom_of(ev), vr_of(ev), e, u, uRec, rhs, scratch, (cudaStream_t)stream);
    if (rc == ST_OK)
        return DNDSB_OK;
    if (rc == ST_NONPHYSICAL)
        return set_error(rc, "dndsb_eval_evaluate_rhs_noalloc: non-physical state (density or pressure <= 0)");
    if (rc == ST_NONFINITE)
        return set_error(rc, "dndsb_eval_evaluate_rhs_noalloc: non-finite value");
    if (rc == ST_UNSUPPORTED)
        return set_error(rc, "dndsb_eval_evaluate_rhs_noalloc: configuration not supported (nVars must be 5 or 6)");
    if (rc == ST_BADARG)
        return set_error(rc, "dndsb_eval_evaluate_rhs_noalloc: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
    return set_error(rc, std::string("dndsb_eval_evaluate_rhs_noalloc: ") + cudaGetErrorString(cudaGetLastError()));
}
