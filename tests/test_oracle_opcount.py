"""The op-counting build of the oracle loads with every entry point it exports, and the algorithmic operation
counts it gives for the TGV workload (python -m oracle.falg) are the F_alg constants the bench reports."""
import bench
import oracle
from oracle import falg


def test_opcount_build_loads():
    L = oracle.opcount_lib()
    assert hasattr(L, "orc_opcount_get") and hasattr(L, "orc_eval_rhs")


def test_falg_constants_match_the_counting_build():
    for p in (2, 1):
        out = falg.tgv(6, p)
        assert out["evaluate_rhs"]["per_cell"] == bench.F_RHS[p], (p, out["evaluate_rhs"]["per_cell"])
        assert out["vr_sweep"]["per_cell"] == bench.F_VR[p], (p, out["vr_sweep"]["per_cell"])
