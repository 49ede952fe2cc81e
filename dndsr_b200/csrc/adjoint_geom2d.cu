// Node-coordinate derivatives of the residual path, 2-D instantiations (VR degree 1 to 3).
// The 3-D instantiations and the host side are in adjoint_geom.cu; both compile the shared
// per-cell recomputation of adjoint_geom.cuh, in two files so that they build in parallel.
#include "adjoint_geom.cuh"

namespace dndsb
{
template void coords_vjp_launch<2>(const MeshD &, const GeomD &, const VRD &, const EulerSettingsD &, const real *, const real *, const real *,
                                   const real *, const real *, const CoordAdjWs &, int *, cudaStream_t);
template void pressure_force_coords_launch<2>(const MeshD &, const GeomD &, const VRD &, real, int, const real *, const real *, const real *,
                                              const CoordAdjWs &, cudaStream_t);
template void coords_jvp_launch<2>(const MeshD &, const GeomD &, const VRD &, const EulerSettingsD &, const real *, const real *,
                                   const real *, const real *, real *, real *, int *, const real *, cudaStream_t);
template void coords_lanes_launch<2>(const MeshD &, const GeomD &, const VRD &, real *, cudaStream_t);
} // namespace dndsb
