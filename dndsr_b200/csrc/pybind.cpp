// pybind11 module dndsr_b200._C: the reference's Python-facing classes (CFV.VariationalReconstruction_2/3,
// src/CFV/VariationalReconstruction_bind.hpp:19-145; the evaluator methods of
// src/CFV/ModelEvaluator_bind.cpp:6-57 on the Euler model) over the C-ABI of include/dndsb.h.
//
// State arrays are torch CUDA tensors, passed by their data pointers after a check of device, dtype
// and contiguity; every call runs on torch's current CUDA stream.  Setup data (mesh arrays, boundary
// tables) are numpy arrays.  A failing call raises dndsr_b200.capi.DndsbError(code, message).
// The module holds no CUDA code: it links libdndsb.so, which must sit next to it.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dndsb.h"

namespace py = pybind11;

namespace
{
[[noreturn]] void raise_status(int rc)
{
    py::object cls = py::module_::import("dndsr_b200.capi").attr("DndsbError");
    py::object exc = cls(rc, std::string(dndsb_last_error()));
    PyErr_SetObject(cls.ptr(), exc.ptr());
    throw py::error_already_set();
}

inline void ck(int rc)
{
    if (rc != DNDSB_OK)
        raise_status(rc);
}

// data pointer of a contiguous CUDA tensor of dtype float64 (or float32); None gives nullptr when allowed
void *dptr(const py::object &t, const char *name, bool fp32 = false, bool nullable = false)
{
    if (t.is_none())
    {
        if (nullable)
            return nullptr;
        throw py::value_error(std::string(name) + " must be a CUDA tensor, not None");
    }
    const char *want = fp32 ? "torch.float32" : "torch.float64";
    if (!py::hasattr(t, "data_ptr") || !t.attr("is_cuda").cast<bool>() || py::str(t.attr("dtype")).cast<std::string>() != want ||
        !t.attr("is_contiguous")().cast<bool>())
        throw py::value_error(std::string(name) + " must be a contiguous " + (fp32 ? "float32" : "float64") + " CUDA tensor");
    return reinterpret_cast<void *>(t.attr("data_ptr")().cast<uintptr_t>());
}
double *dp(const py::object &t, const char *name) { return static_cast<double *>(dptr(t, name)); }
double *dpn(const py::object &t, const char *name) { return static_cast<double *>(dptr(t, name, false, true)); }

// data pointer of any contiguous CUDA tensor
void *anyptr(const py::object &t, const char *name)
{
    if (t.is_none() || !py::hasattr(t, "data_ptr") || !t.attr("is_cuda").cast<bool>() || !t.attr("is_contiguous")().cast<bool>())
        throw py::value_error(std::string(name) + " must be a contiguous CUDA tensor");
    return reinterpret_cast<void *>(t.attr("data_ptr")().cast<uintptr_t>());
}

// 0 for a float64 tensor, 1 for float32
int precision_of(const py::object &t)
{
    std::string d = py::str(t.attr("dtype")).cast<std::string>();
    if (d == "torch.float64")
        return 0;
    if (d == "torch.float32")
        return 1;
    throw py::value_error("Krylov vectors must be float64 or float32");
}

void *stream()
{
    static py::object cur = py::module_::import("torch").attr("cuda").attr("current_stream");
    return reinterpret_cast<void *>(cur().attr("cuda_stream").cast<uintptr_t>());
}

template <class T>
using Arr = py::array_t<T, py::array::c_style | py::array::forcecast>;

struct Mesh
{
    dndsb_mesh *h = nullptr;
    int64_t nCell = 0, nNode = 0;
    Mesh(int dim, int cellType, int faceType, Arr<double> coords, Arr<int64_t> cell2node, Arr<double> cellShift, Arr<int64_t> face2node,
         Arr<double> faceShift, Arr<int64_t> face2cell, Arr<int32_t> faceZone, Arr<double> facePShift, Arr<int64_t> cell2face)
    {
        nNode = coords.shape(0), nCell = cell2node.shape(0);
        ck(dndsb_mesh_create(&h, dim, cellType, faceType, nNode, coords.data(), nCell, (int)cell2node.shape(1), cell2node.data(),
                             cellShift.data(), face2node.shape(0), (int)face2node.shape(1), face2node.data(), faceShift.data(),
                             face2cell.data(), faceZone.data(), facePShift.data(), (int)cell2face.shape(1), cell2face.data()));
    }
    ~Mesh() { dndsb_mesh_destroy(h); }
    py::tuple colors()
    {
        int n = 0;
        Arr<int32_t> col(nCell);
        ck(dndsb_mesh_colors(h, &n, col.mutable_data()));
        return py::make_tuple(n, col);
    }
};

dndsb_vr_settings vr_settings(const py::dict &d)
{
    dndsb_vr_settings s{};
    s.maxOrder = d["maxOrder"].cast<int>(), s.intOrder = d["intOrder"].cast<int>();
    s.jacobiRelax = d["jacobiRelax"].cast<double>(), s.SORInstead = d["SORInstead"].cast<int>();
    s.anisotropicLengths = d["anisotropicLengths"].cast<int>(), s.scaleType = d["scaleType"].cast<int>();
    s.scaleMultiplier = d["scaleMultiplier"].cast<double>(), s.dirWeightScheme = d["dirWeightScheme"].cast<int>();
    auto w = d["manualDirWeights"].cast<std::vector<double>>();
    for (int i = 0; i < 4 && i < (int)w.size(); i++)
        s.manualDirWeights[i] = w[i];
    s.geomWeightScheme = d["geomWeightScheme"].cast<int>(), s.geomWeightBias = d["geomWeightBias"].cast<double>();
    s.geomWeightPower = d["geomWeightPower"].cast<double>(), s.geomWeightPower1 = d["geomWeightPower1"].cast<double>();
    s.geomWeightPower2 = d["geomWeightPower2"].cast<double>(), s.bcWeight = d["bcWeight"].cast<double>();
    return s;
}

dndsb_euler_settings euler_settings(const py::dict &d)
{
    dndsb_euler_settings s{};
    s.nVars = d["nVars"].cast<int>(), s.rsType = d["rsType"].cast<int>();
    s.rsFixScale = d["rsFixScale"].cast<double>(), s.rsIncFScale = d["rsIncFScale"].cast<double>();
    s.gamma = d["gamma"].cast<double>(), s.Rgas = d["Rgas"].cast<double>(), s.muGas = d["muGas"].cast<double>();
    s.prGas = d["prGas"].cast<double>(), s.TRef = d["TRef"].cast<double>(), s.CSutherland = d["CSutherland"].cast<double>();
    s.muModel = d["muModel"].cast<int>(), s.ignoreVis = d["ignoreVis"].cast<int>(), s.rsMeanValueEig = d["rsMeanValueEig"].cast<int>();
    return s;
}

struct VR
{
    dndsb_vr *h = nullptr;
    py::object mesh; // keeps the mesh handle alive
    int64_t nCell = 0, nNode = 0;
    VR(py::object m, const py::dict &settings) : mesh(m)
    {
        Mesh &mm = m.cast<Mesh &>();
        nCell = mm.nCell, nNode = mm.nNode;
        dndsb_vr_settings s = vr_settings(settings);
        ck(dndsb_vr_create(&h, mm.h, &s));
    }
    ~VR() { dndsb_vr_destroy(h); }
    // VariationalReconstruction.cpp:10-43, :56-498, :507-872
    void ConstructMetrics() { ck(dndsb_vr_construct_metrics(h)); }
    void ConstructBaseAndWeight(py::object bcDirWeight)
    {
        if (bcDirWeight.is_none())
            ck(dndsb_vr_construct_base_and_weight(h, nullptr, 0));
        else
        {
            Arr<double> w = bcDirWeight.cast<Arr<double>>();
            ck(dndsb_vr_construct_base_and_weight(h, w.data(), (int)(w.size() / 4)));
        }
    }
    void ConstructRecCoeff() { ck(dndsb_vr_construct_rec_coeff(h)); }
    py::tuple sizes()
    {
        int64_t s[4];
        ck(dndsb_vr_sizes(h, s));
        return py::make_tuple(s[0], s[1], s[2], s[3]);
    }
    Arr<double> get(const std::string &name)
    {
        int64_t n = 0;
        ck(dndsb_vr_get_array(h, name.c_str(), nullptr, 0, &n));
        Arr<double> out(n);
        ck(dndsb_vr_get_array(h, name.c_str(), out.mutable_data(), n, &n));
        return out;
    }
    // VariationalReconstruction_Reconstruction.hxx:485-615
    void DoReconstructionIter(py::object uRec, py::object uRecNew, py::object u, int nVars, bool putIntoNew, bool recordInc, bool uRecIsZero,
                              int precision)
    {
        ck(dndsb_vr_do_reconstruction_iter(h, dp(uRec, "uRec"), dp(uRecNew, "uRecNew"), dp(u, "u"), nVars, putIntoNew, recordInc, uRecIsZero,
                                           precision, stream()));
    }
    void SetBoundary(Arr<int32_t> type, Arr<double> value, int nVars, double gamma, double Rgas)
    {
        ck(dndsb_vr_set_boundary(h, (int)type.size(), type.data(), value.data(), nVars, gamma, Rgas));
    }
    void IterVJP(py::object cot, py::object uRec, py::object u, int nVars, py::object vRec, py::object vU)
    {
        ck(dndsb_vr_iter_vjp(h, dp(cot, "cot"), dp(uRec, "uRec"), dp(u, "u"), nVars, dp(vRec, "vRec"), dp(vU, "vU"), stream()));
    }
    void IterJVP(py::object dRec, py::object du, py::object uRec, py::object u, int nVars, py::object out)
    {
        ck(dndsb_vr_iter_jvp(h, dp(dRec, "dRec"), dp(du, "du"), dp(uRec, "uRec"), dp(u, "u"), nVars, dp(out, "dRecNew"), stream()));
    }
    void IterVJPCoords(py::object cot, py::object uRec, py::object u, int nVars, py::object dX)
    {
        ck(dndsb_vr_iter_vjp_coords(h, dp(cot, "cot"), dp(uRec, "uRec"), dp(u, "u"), nVars, dp(dX, "dX"), stream()));
    }
    void IterJVPCoords(py::object dX, py::object uRec, py::object u, int nVars, py::object out)
    {
        ck(dndsb_vr_iter_jvp_coords(h, dp(dX, "dX"), dp(uRec, "uRec"), dp(u, "u"), nVars, dp(out, "dRecNew"), stream()));
    }
    // VariationalReconstruction_LimiterProcedure.hxx:40-108
    void DoCalculateSmoothIndicator(py::object u, py::object uRec, int nVars, py::object si)
    {
        ck(dndsb_vr_smooth_indicator(h, dp(u, "u"), dp(uRec, "uRec"), nVars, dp(si, "si"), stream()));
    }
};

struct Eval
{
    dndsb_eval *h = nullptr;
    py::object vr;
    int nVars = 5;
    Eval(py::object v, const py::dict &settings) : vr(v)
    {
        dndsb_euler_settings s = euler_settings(settings);
        nVars = s.nVars;
        ck(dndsb_eval_create(&h, v.cast<VR &>().h, &s));
    }
    ~Eval() { dndsb_eval_destroy(h); }
    void SetBC(Arr<int32_t> type, Arr<double> value) { ck(dndsb_eval_set_bc(h, (int)type.size(), type.data(), value.data())); }
    void SetWallDistance(Arr<double> d) { ck(dndsb_eval_set_wall_distance(h, d.data())); }
    void InitializeUDOF(py::object u, int kind, double chi) { ck(dndsb_eval_initialize_udof(h, kind, chi, dp(u, "u"), stream())); }
    // EulerEvaluator_EvaluateDt.hxx:840-1048
    py::object EvaluateDt(py::object dt, py::object u, double CFL, double MaxDt, bool useLocalDt, bool wantMin)
    {
        double mn = 0;
        bool ask = wantMin || !useLocalDt;
        ck(dndsb_eval_evaluate_dt(h, dp(u, "u"), CFL, MaxDt, useLocalDt, dp(dt, "dt"), ask ? &mn : nullptr, stream()));
        return ask ? py::object(py::float_(mn)) : py::object(py::none());
    }
    // EulerEvaluator_EvaluateRHS.hxx:55-818
    void EvaluateRHS(py::object rhs, py::object u, py::object uRec)
    {
        ck(dndsb_eval_evaluate_rhs(h, dp(rhs, "rhs"), dp(u, "u"), dp(uRec, "uRec"), stream()));
    }
    void EvaluateRHSFull(py::object rhs, py::object JSource, py::object u, py::object uRecUnlim, py::object uRec, py::object uRecBeta,
                         py::object cellRHSAlpha, bool onlyOnHalfAlpha, double t, uint64_t flags)
    {
        ck(dndsb_eval_evaluate_rhs_full(h, dp(rhs, "rhs"), dpn(JSource, "JSource"), dp(u, "u"), dp(uRecUnlim, "uRecUnlim"), dp(uRec, "uRec"),
                                        dpn(uRecBeta, "uRecBeta"), dpn(cellRHSAlpha, "cellRHSAlpha"), onlyOnHalfAlpha, t, flags, stream()));
    }
    void EvaluateRHSNoAlloc(py::object rhs, py::object u, py::object uRec)
    {
        ck(dndsb_eval_evaluate_rhs_noalloc(h, dp(rhs, "rhs"), dp(u, "u"), dp(uRec, "uRec"), stream()));
    }
    void SetDeferredErrors(bool on) { ck(dndsb_eval_set_deferred_errors(h, on)); }
    void CheckErrors() { ck(dndsb_eval_check_errors(h, stream())); }
    void RhsVJP(py::object w, py::object u, py::object uRec, py::object du, py::object duRec)
    {
        ck(dndsb_eval_rhs_vjp(h, dp(w, "w"), dp(u, "u"), dp(uRec, "uRec"), dp(du, "du"), dp(duRec, "duRec"), stream()));
    }
    void WallFluxVJP(Arr<double> dir, py::object u, py::object uRec, py::object du, py::object duRec)
    {
        ck(dndsb_eval_wall_flux_vjp(h, dir.data(), dp(u, "u"), dp(uRec, "uRec"), dp(du, "du"), dp(duRec, "duRec"), stream()));
    }
    void RhsJVP(py::object du, py::object duRec, py::object u, py::object uRec, py::object out)
    {
        ck(dndsb_eval_rhs_jvp(h, dp(du, "du"), dp(duRec, "duRec"), dp(u, "u"), dp(uRec, "uRec"), dp(out, "dRhs"), stream()));
    }
    void RhsVJPCoords(py::object w, py::object u, py::object uRec, py::object dX)
    {
        ck(dndsb_eval_rhs_vjp_coords(h, dp(w, "w"), dp(u, "u"), dp(uRec, "uRec"), dp(dX, "dX"), stream()));
    }
    void ResidualVJPCoords(py::object w, py::object cot, py::object u, py::object uRec, py::object dX)
    {
        ck(dndsb_eval_residual_vjp_coords(h, dp(w, "w"), dp(cot, "cot"), dp(u, "u"), dp(uRec, "uRec"), dp(dX, "dX"), stream()));
    }
    void RhsJVPCoords(py::object dX, py::object u, py::object uRec, py::object out)
    {
        ck(dndsb_eval_rhs_jvp_coords(h, dp(dX, "dX"), dp(u, "u"), dp(uRec, "uRec"), dp(out, "dRhs"), stream()));
    }
    // EulerEvaluator.hxx:37-159, :175-274, :376-529, :550-693
    void LUSGSMatrixInit(py::object jd, py::object dTau, double dt, double alphaDiag)
    {
        ck(dndsb_eval_lusgs_matrix_init(h, dp(dTau, "dTau"), dt, alphaDiag, dp(jd, "jdiag"), stream()));
    }
    void LUSGSMatrixInitFull(py::object jd, py::object dTau, double dt, double alphaDiag, py::object u, py::object uRec, int jacobianCode, double t)
    {
        ck(dndsb_eval_lusgs_matrix_init_full(h, dp(dTau, "dTau"), dt, alphaDiag, dpn(u, "u"), dpn(uRec, "uRec"), jacobianCode, t, dp(jd, "jdiag"),
                                             stream()));
    }
    void SetJacobianMode(bool useScalarJacobian, bool useRoeJacobian) { ck(dndsb_eval_set_jacobian_mode(h, useScalarJacobian, useRoeJacobian)); }
    // EulerEvaluator.hxx:290-359, 838-927
    void LUSGSMatrixToJacobianLU(double alphaDiag, py::object u, py::object jd)
    {
        ck(dndsb_eval_lusgs_matrix_to_jacobian_lu(h, alphaDiag, dp(u, "u"), dp(jd, "jdiag"), stream()));
    }
    py::object LUSGSMatrixSolveJacobianLU(double alphaDiag, py::object rhs, py::object u, py::object uInc, py::object uIncNew, py::object jd,
                                          bool uIncIsZero, bool wantSum)
    {
        Arr<double> s(nVars);
        ck(dndsb_eval_lusgs_matrix_solve_jacobian_lu(h, alphaDiag, dp(rhs, "rhs"), dp(u, "u"), dp(uInc, "uInc"), dp(uIncNew, "uIncNew"),
                                                     dp(jd, "jdiag"), uIncIsZero, wantSum ? s.mutable_data() : nullptr, stream()));
        return wantSum ? py::object(s) : py::object(py::none());
    }
    py::object UpdateSGS(double alphaDiag, py::object rhs, py::object u, py::object uInc, py::object uIncNew, py::object jd, bool forward,
                         bool gsUpdate, bool uIncIsZero, bool wantSum)
    {
        Arr<double> s(nVars);
        ck(dndsb_eval_update_sgs(h, alphaDiag, dp(rhs, "rhs"), dp(u, "u"), dp(uInc, "uInc"), dp(uIncNew, "uIncNew"), dp(jd, "jdiag"), forward,
                                 gsUpdate, uIncIsZero, wantSum ? s.mutable_data() : nullptr, stream()));
        return wantSum ? py::object(s) : py::object(py::none());
    }
    void UpdateLUSGSForward(double alphaDiag, py::object rhs, py::object u, py::object uInc, py::object jd, py::object uIncNew)
    {
        ck(dndsb_eval_update_lusgs_forward(h, alphaDiag, dp(rhs, "rhs"), dp(u, "u"), dp(uInc, "uInc"), dp(jd, "jdiag"), dp(uIncNew, "uIncNew"),
                                           stream()));
    }
    void UpdateLUSGSBackward(double alphaDiag, py::object rhs, py::object u, py::object uInc, py::object jd, py::object uIncNew)
    {
        ck(dndsb_eval_update_lusgs_backward(h, alphaDiag, dp(rhs, "rhs"), dp(u, "u"), dp(uInc, "uInc"), dp(jd, "jdiag"), dp(uIncNew, "uIncNew"),
                                            stream()));
    }
    void FixUMaxFilter(py::object u) { ck(dndsb_eval_fix_umax_filter(h, dp(u, "u"), stream())); }
    void LUSGSMatrixVec(double alphaDiag, py::object u, py::object uInc, py::object jd, py::object Au)
    {
        ck(dndsb_eval_lusgs_matrix_vec(h, alphaDiag, dp(u, "u"), dp(uInc, "uInc"), dp(jd, "jdiag"), dp(Au, "AuInc"), stream()));
    }
    void LUSGSMatrixVecT(double alphaDiag, py::object u, py::object y, py::object jd, py::object ATy)
    {
        ck(dndsb_eval_lusgs_matrix_vec_t(h, alphaDiag, dp(u, "u"), dp(y, "y"), dp(jd, "jdiag"), dp(ATy, "ATy"), stream()));
    }
    void UpdateSGST(double alphaDiag, py::object b, py::object u, py::object y, py::object yNew, py::object jd, bool forward, bool gsUpdate,
                    bool fp32)
    {
        ck(dndsb_eval_update_sgs_t(h, alphaDiag, dptr(b, "b", fp32), dp(u, "u"), dptr(y, "y", fp32), dptr(yNew, "yNew", fp32), dp(jd, "jdiag"),
                                   forward, gsUpdate, fp32, stream()));
    }
    double PressureForce(int zone, Arr<double> dir, py::object u, py::object uRec, py::object dJdu, py::object dJduRec)
    {
        double J = 0;
        ck(dndsb_eval_pressure_force(h, zone, dir.data(), dp(u, "u"), dp(uRec, "uRec"), &J, dpn(dJdu, "dJdu"), dpn(dJduRec, "dJduRec"),
                                     stream()));
        return J;
    }
    void PressureForceCoords(int zone, Arr<double> dir, py::object u, py::object uRec, py::object dX)
    {
        ck(dndsb_eval_pressure_force_coords(h, zone, dir.data(), dp(u, "u"), dp(uRec, "uRec"), dp(dX, "dJdX"), stream()));
    }
    void DoLimiterWBAP_C(py::object u, py::object uRec, py::object si, py::object uRecNew, double thr, double nStd, bool ifAll)
    {
        ck(dndsb_eval_limiter_wbap_c(h, dp(u, "u"), dp(uRec, "uRec"), dp(si, "si"), dp(uRecNew, "uRecNew"), thr, nStd, ifAll, stream()));
    }
    py::tuple EvaluateCellRHSAlpha(py::object u, py::object res, py::object alpha, double refRho, double refP, double relax, int compress,
                                   double compressPower, bool ppEpsIsRelaxed, int flag)
    {
        int64_t n = 0;
        double amin = 0;
        ck(dndsb_eval_cell_rhs_alpha(h, dp(u, "u"), dp(res, "res"), dp(alpha, "alpha"), refRho, refP, relax, compress, compressPower,
                                     ppEpsIsRelaxed, flag, &n, &amin, stream()));
        return py::make_tuple(n, amin);
    }
    void EvaluateCellRHSAlphaExpansion(py::object u, py::object res, py::object alpha, double refRho, double refP, double alphaMin)
    {
        ck(dndsb_eval_cell_rhs_alpha_expansion(h, dp(u, "u"), dp(res, "res"), dp(alpha, "alpha"), refRho, refP, alphaMin, stream()));
    }
    double AddFixedIncrement(py::object u, py::object inc, double alpha, double refRho, double refP, bool ppEpsIsRelaxed)
    {
        double amin = 0;
        ck(dndsb_eval_add_fixed_increment(h, dp(u, "u"), dp(inc, "inc"), alpha, refRho, refP, ppEpsIsRelaxed, &amin, stream()));
        return amin;
    }
    // EulerSolver.hxx:1407-1658 with Solver/Linear.hpp:46-133
    void SolveLinear(const py::dict &ls, double alphaDiag, py::object dTau, double dt, py::object u, py::object rhs, py::object xInc)
    {
        dndsb_linear_settings s{};
        s.gmresCode = ls["gmresCode"].cast<int>(), s.jacobiCode = ls["jacobiCode"].cast<int>(), s.sgsIter = ls["sgsIter"].cast<int>();
        s.nGmresSpace = ls["nGmresSpace"].cast<int>(), s.nGmresIter = ls["nGmresIter"].cast<int>();
        s.precision = ls["precision"].cast<int>(), s.useGraph = ls["useGraph"].cast<int>();
        auto ms = ls["meanScale"].cast<std::vector<double>>();
        for (int i = 0; i < 8 && i < (int)ms.size(); i++)
            s.meanScale[i] = ms[i];
        ck(dndsb_eval_solve_linear(h, &s, alphaDiag, dp(dTau, "dTau"), dt, dp(u, "u"), dp(rhs, "rhs"), dp(xInc, "xInc"), stream()));
    }
    // EulerEvaluator.hxx:1394-1439
    Arr<double> EvaluateNorm(py::object x, int P, bool volWise)
    {
        Arr<double> out(nVars);
        ck(dndsb_eval_evaluate_norm(h, dp(x, "x"), P, volWise, out.mutable_data(), stream()));
        return out;
    }
    Arr<double> get(const std::string &name)
    {
        int64_t n = 0;
        ck(dndsb_eval_get_array(h, name.c_str(), nullptr, 0, &n));
        Arr<double> out(n);
        ck(dndsb_eval_get_array(h, name.c_str(), out.mutable_data(), n, &n));
        return out;
    }
    void SetDeltaLambda(py::object dl) { ck(dndsb_eval_set_delta_lambda(h, dp(dl, "deltaLambdaCell"), stream())); }
};
} // namespace

PYBIND11_MODULE(_C, m)
{
    m.doc() = "B200 implementation of DNDSR's implicit residual path: mesh, variational reconstruction and Euler "
              "evaluator handles over the C-ABI of include/dndsb.h";
    m.def("version", &dndsb_version);
    // device Krylov primitives of a caller-driven GMRES (include/dndsb.h); V [k+1][krylov_ld(n)] zero-filled
    m.def("krylov_ld", &dndsb_krylov_ld);
    m.def("krylov_work_bytes", &dndsb_krylov_work_bytes);
    m.def("krylov_start",
          [](py::object r, py::object V, py::object gsc, py::object colScale, py::object work, int k)
          {
              const int prec = precision_of(V);
              ck(dndsb_krylov_start(prec, r.attr("numel")().cast<int64_t>(), k, dptr(r, "r", prec == 1), anyptr(V, "V"), dp(gsc, "gsc"),
                                    dp(colScale, "colScale"), anyptr(work, "work"), stream()));
          });
    m.def("krylov_arnoldi",
          [](int64_t n, int j, int k, py::object V, py::object H, py::object colScale, py::object gsc, py::object res, py::object work)
          {
              ck(dndsb_krylov_arnoldi(precision_of(V), n, j, k, anyptr(V, "V"), dp(H, "H"), dp(colScale, "colScale"), dp(gsc, "gsc"),
                                      dpn(res, "res"), anyptr(work, "work"), stream()));
          });
    m.def("krylov_update",
          [](int64_t n, int k, py::object V, py::object gsc, py::object colScale, py::object x)
          {
              const int prec = precision_of(V);
              ck(dndsb_krylov_update(prec, n, k, anyptr(V, "V"), dp(gsc, "gsc"), dp(colScale, "colScale"), dptr(x, "x", prec == 1), stream()));
          });
    py::class_<Mesh>(m, "Mesh")
        .def(py::init<int, int, int, Arr<double>, Arr<int64_t>, Arr<double>, Arr<int64_t>, Arr<double>, Arr<int64_t>, Arr<int32_t>,
                      Arr<double>, Arr<int64_t>>(),
             py::arg("dim"), py::arg("cellType"), py::arg("faceType"), py::arg("coords"), py::arg("cell2node"), py::arg("cellShift"),
             py::arg("face2node"), py::arg("faceShift"), py::arg("face2cell"), py::arg("faceZone"), py::arg("facePShift"),
             py::arg("cell2face"))
        .def("colors", &Mesh::colors);
    auto vr = py::class_<VR>(m, "VariationalReconstruction")
                  .def(py::init<py::object, const py::dict &>(), py::arg("mesh"), py::arg("settings"))
                  .def("ConstructMetrics", &VR::ConstructMetrics)
                  .def("ConstructBaseAndWeight", &VR::ConstructBaseAndWeight, py::arg("bcDirWeight") = py::none())
                  .def("ConstructRecCoeff", &VR::ConstructRecCoeff)
                  .def("sizes", &VR::sizes)
                  .def("get", &VR::get)
                  .def("DoReconstructionIter", &VR::DoReconstructionIter, py::arg("uRec"), py::arg("uRecNew"), py::arg("u"), py::arg("nVars"),
                       py::arg("putIntoNew"), py::arg("recordInc"), py::arg("uRecIsZero"), py::arg("precision") = 0)
                  .def("SetBoundary", &VR::SetBoundary)
                  .def("DoReconstructionIterVJP", &VR::IterVJP)
                  .def("DoReconstructionIterJVP", &VR::IterJVP)
                  .def("DoReconstructionIterVJPCoords", &VR::IterVJPCoords)
                  .def("DoReconstructionIterJVPCoords", &VR::IterJVPCoords)
                  .def("DoCalculateSmoothIndicator", &VR::DoCalculateSmoothIndicator);
    // the reference binds one class per dimension; the dimension here is a property of the mesh
    m.attr("VariationalReconstruction_2") = vr;
    m.attr("VariationalReconstruction_3") = vr;
    py::class_<Eval>(m, "EulerEvaluator")
        .def(py::init<py::object, const py::dict &>(), py::arg("vfv"), py::arg("settings"))
        .def_readonly("nVars", &Eval::nVars)
        .def("SetBC", &Eval::SetBC)
        .def("SetWallDistance", &Eval::SetWallDistance)
        .def("InitializeUDOF", &Eval::InitializeUDOF)
        .def("EvaluateDt", &Eval::EvaluateDt)
        .def("EvaluateRHS", &Eval::EvaluateRHS)
        .def("EvaluateRHSFull", &Eval::EvaluateRHSFull)
        .def("EvaluateRHSNoAlloc", &Eval::EvaluateRHSNoAlloc)
        .def("SetDeferredErrors", &Eval::SetDeferredErrors)
        .def("CheckErrors", &Eval::CheckErrors)
        .def("EvaluateRHSVJP", &Eval::RhsVJP)
        .def("EvaluateRHSJVP", &Eval::RhsJVP)
        .def("WallFluxVJP", &Eval::WallFluxVJP)
        .def("EvaluateRHSVJPCoords", &Eval::RhsVJPCoords)
        .def("ResidualVJPCoords", &Eval::ResidualVJPCoords)
        .def("EvaluateRHSJVPCoords", &Eval::RhsJVPCoords)
        .def("LUSGSMatrixInit", &Eval::LUSGSMatrixInit)
        .def("LUSGSMatrixInitFull", &Eval::LUSGSMatrixInitFull)
        .def("SetJacobianMode", &Eval::SetJacobianMode)
        .def("LUSGSMatrixToJacobianLU", &Eval::LUSGSMatrixToJacobianLU)
        .def("LUSGSMatrixSolveJacobianLU", &Eval::LUSGSMatrixSolveJacobianLU)
        .def("UpdateSGS", &Eval::UpdateSGS)
        .def("UpdateLUSGSForward", &Eval::UpdateLUSGSForward)
        .def("UpdateLUSGSBackward", &Eval::UpdateLUSGSBackward)
        .def("FixUMaxFilter", &Eval::FixUMaxFilter)
        .def("LUSGSMatrixVec", &Eval::LUSGSMatrixVec)
        .def("LUSGSMatrixVecT", &Eval::LUSGSMatrixVecT)
        .def("UpdateSGST", &Eval::UpdateSGST)
        .def("PressureForce", &Eval::PressureForce)
        .def("PressureForceCoords", &Eval::PressureForceCoords)
        .def("DoLimiterWBAP_C", &Eval::DoLimiterWBAP_C)
        .def("EvaluateCellRHSAlpha", &Eval::EvaluateCellRHSAlpha)
        .def("EvaluateCellRHSAlphaExpansion", &Eval::EvaluateCellRHSAlphaExpansion)
        .def("AddFixedIncrement", &Eval::AddFixedIncrement)
        .def("SolveLinear", &Eval::SolveLinear)
        .def("EvaluateNorm", &Eval::EvaluateNorm)
        .def("get", &Eval::get)
        .def("SetDeltaLambda", &Eval::SetDeltaLambda);
}
