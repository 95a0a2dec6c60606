"""The tcgen05 tensor-core GEMM kinds (TF32 and 3xBF16) against FP64.

The precision form of the block GEMMs: FP64 in and out, reduced arithmetic inside.  The
bounds are written as relative Frobenius errors: TF32 keeps 11 significand bits of each
operand (error ~ 2^-11), the 3xBF16 split keeps ~16 (error ~ 2^-16), both with FP32
accumulation.
"""

import numpy as np
import pytest
import torch

import oracle.tenet_oracle as O
from tenet import _exec, _lib

pytestmark = pytest.mark.gpu

TOL = {3: 5e-3, 4: 5e-5}


@pytest.fixture(autouse=True)
def _device_error_clear():
    yield
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0, "a kernel raised the device error word"


@pytest.mark.parametrize("kind", [3, 4])
def test_tensorcore_gemm_kinds(kind):
    rng = np.random.default_rng(kind)
    shapes = [(176, 236, 60), (9, 11, 2), (300, 200, 500), (40, 7, 0), (128, 64, 32),
              (129, 65, 33), (1, 1, 1)]
    a_off = b_off = c_off = 0
    prods, offs = [], []
    for M, N, K in shapes:
        prods.append((M, N, K, a_off, K, b_off, N, c_off, N))
        offs.append((a_off, b_off, c_off))
        a_off += M * K
        b_off += K * N
        c_off += M * N
    A, B = rng.standard_normal(a_off), rng.standard_normal(b_off)
    table = _exec.make_gemm(prods, kind)
    ta, tb = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    for _ in range(2):
        tc = torch.full((c_off,), float("nan"), dtype=torch.float64, device="cuda")
        table.run(ta, tb, tc)
        C = tc.cpu().numpy()
        for (M, N, K), (ao, bo, co) in zip(shapes, offs):
            want = A[ao:ao + M * K].reshape(M, K) @ B[bo:bo + K * N].reshape(K, N)
            got = C[co:co + M * N].reshape(M, N)
            assert not np.isnan(got).any()
            if K == 0:
                assert (got == 0).all()
                continue
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err < TOL[kind], f"{(M, N, K)}: relative error {err:.2e}"


@pytest.mark.parametrize("precision,tol,tc_min", [("3xbf16", 1e-4, None), ("tf32", 1e-2, None),
                                                  ("3xbf16", 1e-4, 0), ("tf32", 1e-2, 0)])
def test_mixed_precision_heff2_chain(precision, tol, tc_min):
    """The bench's large-bond SU(2) matvec (256 multiplets) with its big sector products
    (or, with ``tc_min`` 0, all of them) on the tensor cores, in the reference's order and
    in the folded form."""
    import bench
    from tenet import network
    from tenet.program import heff2_folded_program, heff2_program

    tensors = bench.build_workload(bond=bench.WORKLOADS["synthetic_256_multiplets"])
    fl, w1, w2, fr, aa = tensors
    lf, rf = network.fold_left(fl, w1), network.fold_right(w2, fr)
    folded = heff2_folded_program(lf, rf, aa.structure, precision=precision,
                                  tc_min_flops=tc_min)
    assert folded.uses_tensor_cores
    exact = heff2_program(*tensors[:4], tensors[4].structure)(tensors[4]).numpy_arena()
    prog = heff2_program(*tensors[:4], tensors[4].structure, precision=precision,
                         tc_min_flops=tc_min)
    assert prog.uses_tensor_cores
    for p in (prog, folded):
        got = p(tensors[4]).numpy_arena()
        err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
        assert err < tol, f"{precision}: relative error {err:.2e}"


@pytest.mark.parametrize("precision", ["3xbf16"])
def test_mixed_precision_dmrg_energy(golden_dir, precision):
    """DMRG with tensor-core matvecs and the FP64 correction: |dE/L| <= 1e-8 against the
    reference's FP64 run (SU(2) Heisenberg L = 16, chi = 24, ncv = 20)."""
    import json

    from tenet import network
    from tenet.structure import GradedSpace
    from tenet.symmetry import SU2

    g = json.loads((golden_dir / "dmrg.json").read_text())["L16_chi24"]
    L, chi = g["L"], g["chi"]
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    e = network.dmrg_(network.MPS.random(phys, bonds, seed=0),
                      network.heisenberg_mpo_su2(L), chi=chi, cutoff=1e-10, ncv=20,
                      max_sweeps=g["sweeps"], energy_tol=0.0, precision=precision,
                      tc_min_flops=0).energy  # every product on the tensor cores
    assert abs(e - g["energy"]) / L <= 1e-8, f"|dE/L| = {abs(e - g['energy']) / L:.2e}"


@pytest.mark.parametrize("precision,rel", [("3xbf16", 1e-10), ("tf32", 1e-7)])
def test_mixed_precision_ctmrg_free_energy(golden_dir, precision, rel):
    """Z2 Ising CTMRG with every corner / edge sector product on the tensor cores (the SVD
    and truncation in FP64): the free energy against the reference's converged FP64 run
    (beta = 0.4, chi = 16) and the even/odd bond split unchanged."""
    import json

    import oracle.tenet_oracle as O
    from tenet import network

    r = json.loads((golden_dir / "ctmrg.json").read_text())["b040_chi16"]
    bulk = network.ising_bulk(r["beta"])
    c, e, bond, _ = network.ctmrg(*network.single_layer_ctm(bulk), chi=r["chi"], tol=r["tol"],
                                  max_sweeps=r["max_sweeps"], precision=precision,
                                  tc_min_flops=0)
    bf = network.beta_free_energy(c, e, bulk)
    assert abs(bf - r["beta_f"]) <= rel * abs(r["beta_f"])
    assert abs(bf - O.onsager_beta_f(r["beta"])) <= max(rel, 1e-9) * abs(r["beta_f"])
    assert [[a.parity, m] for a, m in bond.sectors] == r["bond"]


def test_mixed_precision_ctmrg_chi128_near_criticality():
    """beta = 0.44, chi = 128 (the even/odd split 64/64), 150 moves: 3xBF16 corner and edge
    products give the FP64 free energy to 1e-8, both within 1e-6 of Onsager's (the bound
    of the reference's own CTMRG test; near criticality 150 moves are not converged)."""
    import oracle.tenet_oracle as O
    from tenet import network

    bulk = network.ising_bulk(0.44)
    out = {}
    for prec in ("f64", "3xbf16"):
        c, e, bond, _ = network.ctmrg(*network.single_layer_ctm(bulk), chi=128, tol=1e-10,
                                      max_sweeps=150, precision=prec, tc_min_flops=0)
        out[prec] = network.beta_free_energy(c, e, bulk)
        assert [m for _, m in bond.sectors] == [64, 64]
    assert abs(out["3xbf16"] - out["f64"]) <= 1e-8 * abs(out["f64"])
    assert abs(out["3xbf16"] - O.onsager_beta_f(0.44)) <= 1e-6 * abs(out["f64"])


@pytest.mark.parametrize("precision", ["3xbf16", "tf32"])
def test_residual_correction_of_the_precision_lanczos_vector(golden_dir, precision):
    """The precision form's FP64 residual correction (``DeviceLanczos._residual_step``) on
    the reference's converged L = 12 mid-bond operator with every non-skinny product on
    the tensor cores: the reduced-precision Ritz vector's FP64 residual drops by more than
    an order of magnitude and the energy moves to the FP64 solve's."""
    import json

    from tenet import network, ops
    from tenet.program import heff2_folded_program
    from tenet.structure import TensorStructure  # noqa: F401

    from test_gpu_parity import load

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    lf, rf = network.fold_left(T["fl"], T["w1"]), network.fold_right(T["w2"], T["fr"])
    aa = T["aa"]
    p64 = heff2_folded_program(lf, rf, aa.structure)
    ptc = heff2_folded_program(lf, rf, aa.structure, precision=precision, tc_min_flops=0)
    assert ptc.uses_tensor_cores

    def residual(v):
        hv = p64(v)
        theta = ops.inner(v, hv)
        return ops.norm(ops.subtract(hv, v * theta)) / abs(theta)

    e64, v64 = network.DeviceLanczos(p64, 20).solve(aa)
    e1, v1 = network.DeviceLanczos(ptc, 20, correct=p64, residual=False).solve(aa)
    e2, v2 = network.DeviceLanczos(ptc, 20, correct=p64, residual=True).solve(aa)
    r64, r1, r2 = residual(v64), residual(v1), residual(v2)
    assert r64 < 1e-9  # the operator is converged at ncv = 20 in FP64
    assert r2 < 0.1 * r1, (r1, r2)
    assert abs(e2 - e64) <= abs(e1 - e64) + 1e-13 * abs(e64)
    assert abs(ops.norm(v2) - 1.0) < 1e-12
