"""Host-side logic and the C ABI surface (no GPU needed)."""
import ctypes
import importlib

import numpy as np
import pytest


def test_library_exports_header(hx):
    L = importlib.import_module("2025_12_09_hexat_v069_b200._lib")
    lib = L.load()
    syms = L.header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(L.PROTOTYPES)


def test_abi_struct_sizes(hx):
    L = importlib.import_module("2025_12_09_hexat_v069_b200._lib")
    # natural x86-64 alignment, identical for the C compiler and ctypes
    assert ctypes.sizeof(L.SolveOpts) == 96
    assert ctypes.sizeof(L.SolveReport) == 6 * 4 + 10 * 8
    assert ctypes.sizeof(L.UpdateParams) == 176
    assert ctypes.sizeof(L.UpdateResult) == 64


def test_no_device_fails_loudly(hx):
    """Without a GPU, context creation returns a status; nothing runs on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hx.HexatError) as e:
        hx.Context(0)
    assert e.value.status in (8, 7)


def test_generate_mesh_layout(hx):
    nodes, el, dims = hx.mesh.generate_mesh(3, 2, 2)
    assert dims == (4, 3, 3)
    assert nodes.shape == (36, 3) and el.shape == (12, 8)
    # node_index(i,j,k) = i + (j-1)nx + (k-1)nx ny (Mesh.jl:13-15), 1-based
    assert hx.mesh.node_index(2, 3, 2, 4, 3) == 2 + 2 * 4 + 1 * 12
    assert list(nodes[hx.mesh.node_index(2, 3, 2, 4, 3) - 1]) == [1.0, 2.0, 1.0]
    # element 1 corners follow NAT_COORDS
    e = el[0] - 1
    want = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    assert [tuple(nodes[n]) for n in e] == want
    # element numbering i fastest
    assert el[1, 0] == 2 and el[3, 0] == 5


def test_location_grammar(hx):
    nodes, _, _ = hx.mesh.generate_mesh(60, 20, 20)
    B = hx.boundary
    # 60 > 1: absolute; 10 > 1: absolute (the C0 load line)
    sel = B.nodes_by_location([60, ":", 10], nodes)
    assert len(sel) == 21 and np.all(nodes[sel, 0] == 60) and np.all(nodes[sel, 2] == 10)
    # a number in [0,1] is a FRACTION of the extent (Boundary.jl:119-120)
    sel1 = B.nodes_by_location([1, ":", ":"], nodes)
    assert np.all(nodes[sel1, 0] == 60)
    sel05 = B.nodes_by_location([0.5, ":", ":"], nodes)
    assert np.all(nodes[sel05, 0] == 30)
    selp = B.nodes_by_location(["25%", 0, ":"], nodes)
    assert np.all(nodes[selp, 0] == 15) and np.all(nodes[selp, 1] == 0)
    bc = B.get_bc_indicator(nodes.shape[0], nodes, [{"location": [0, ":", ":"], "DoFs": [1, 2, 3]}])
    assert bc.sum() == 3 * 21 * 21
    F = np.zeros(3 * nodes.shape[0])
    B.apply_external_forces(F, [{"location": [60, ":", 10], "F": [0, -1, 0]}], nodes)
    assert F.sum() == pytest.approx(-1.0) and np.count_nonzero(F) == 21
    # a point spec that matches nothing maps to the nearest node
    F2 = np.zeros(3 * nodes.shape[0])
    B.apply_external_forces(F2, [{"location": [59.6, 19.7, 10.2], "F": [1, 0, 0]}], nodes)
    n = np.nonzero(F2)[0][0] // 3
    assert list(nodes[n]) == [60.0, 20.0, 10.0]
    with pytest.raises(ValueError):
        B.get_bc_indicator(nodes.shape[0], nodes, [{"location": [0, ":", ":"], "DoFs": [4]}])


def test_splitmix_known_answers(hx):
    u = hx.workloads.splitmix64_uniform(20251209, 4)
    v = hx.workloads.splitmix64_uniform(20251209, 2, offset=2)
    assert np.array_equal(u[2:], v)
    assert np.all((u >= 0) & (u < 1))
    # fixed values of the counter-based generator (regression pins)
    ref = hx.workloads.splitmix64_uniform(0, 1)[0]
    z = (0x9E3779B97F4A7C15 * 1) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    z ^= z >> 31
    assert ref == (z >> 11) / 2.0 ** 53


def test_cantilever_and_mbb(hx):
    nodes, el, bc, f = hx.workloads.cantilever(60, 20, 20)
    assert f.sum() == pytest.approx(-1.0) and np.count_nonzero(f) == 21
    assert bc.sum() == 3 * 21 * 21
    n2, _, bc2, f2 = hx.workloads.cantilever(60, 20, 20, with_elements=False)
    assert np.array_equal(f, f2) and np.array_equal(bc, bc2)
    nodes, el, bc, f = hx.workloads.mbb_half_beam(12, 4, 4)
    assert bc[:, 0].sum() == 5 * 5 and bc[:, 1].sum() == 5 and bc[:, 2].sum() == 0
    assert f.sum() == pytest.approx(-1.0)


def test_noalloc_rejects_bad_arguments_before_the_device(hx):
    """hx_apply_stiffness_noalloc checks its arguments before any CUDA call:
    misaligned pointers and grids beyond the kernels' index range return
    HX_BAD_ARG (6).  Run where no GPU is present, so the pointers (host
    buffers) can never reach a kernel even if a check were missing; on a GPU
    machine the device-pointer form of this test runs with the GPU tests."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: covered by the no-alloc GPU test")
    L = importlib.import_module("2025_12_09_hexat_v069_b200._lib")
    lib = L.load()
    buf = np.zeros(64, np.float64)
    p = buf.ctypes.data
    assert p % 16 == 0
    good = (p, p + 128, p + 256, p + 384)
    for k, off in ((0, 8), (1, 4), (2, 4), (3, 4)):
        args = list(good)
        args[k] += off
        assert lib.hx_apply_stiffness_noalloc(2, 2, 2, 1.0, 1.0, 1.0, 0.3, *args, None) == 6
    # 3 x nodes per z-plane at 2^31 and beyond: in-plane offsets would overflow
    assert lib.hx_apply_stiffness_noalloc(30000, 30000, 1, 1.0, 1.0, 1.0, 0.3, *good, None) == 6
    assert lib.hx_apply_stiffness_noalloc(1 << 20, 1, 1, 1.0, 1.0, 1.0, 0.3, *good, None) == 6
    assert lib.hx_apply_stiffness_noalloc(0, 1, 1, 1.0, 1.0, 1.0, 0.3, *good, None) == 6
    assert lib.hx_apply_stiffness_noalloc(2, 2, 2, 1.0, 1.0, 1.0, 0.5, *good, None) == 6
    # valid arguments get as far as the device query, which fails without a GPU
    assert lib.hx_apply_stiffness_noalloc(2, 2, 2, 1.0, 1.0, 1.0, 0.3, *good, None) in (7, 8)


def test_update_params_from_reference_config(hx):
    """The config Dict keys update_density! reads (TopOpt.jl:156-169, 216-222,
    351-352) and its defaults, packed for hx_update_density."""
    api = importlib.import_module("2025_12_09_hexat_v069_b200.api")
    cfg = {"geometry": {"nElem_x_computed": 60, "nElem_y_computed": 20, "nElem_z_computed": 20,
                        "dx_computed": 1.0, "dy_computed": 1.0, "dz_computed": 1.0,
                        "max_domain_dim": 60.0},
           "optimization_parameters": {"filter_R_init_perc": 4.0, "max_culling_ratio": 0.05}}
    p = api.update_params(cfg)
    assert list(p.nelem) == [60, 20, 20] and p.max_domain_dim == 60.0
    assert p.filter_R_init_perc == 4.0 and p.filter_R_interm_iter_perc == 50.0
    assert p.final_density_threshold == 0.95 and p.max_culling_ratio == 0.05
    assert p.filter_tolerance == 1e-5 and p.mode == 0
    cfg["optimization_parameters"]["update"] = "oc"
    assert api.update_params(cfg).mode == 1
    cfg["optimization_parameters"]["update"] = "bogus"
    with pytest.raises(ValueError):
        api.update_params(cfg)


def test_reference_preconditioner_config_maps_to_dropin_solver():
    """The reference's solver_parameters.preconditioner values select the
    drop-in solver (src/Solvers/GPUSolver.jl:320-324): jacobi, jacobi_amg
    (Jacobi with the multigrid fallback), amg (multigrid from the start);
    no key leaves the context's choice; an unknown name is an error."""
    import importlib
    api = importlib.import_module("2025_12_09_hexat_v069_b200.api")

    class Fake:
        calls = []

        def set_dropin_solver(self, *a):
            self.calls.append(a)

    ctx = Fake()
    for name, want in [("Jacobi", (0, 0, 0)), ("jacobi_amg", (0, 0, 1)), ("AMG", (3, 0, 0))]:
        api._apply_solver_config(ctx, {"solver_parameters": {"preconditioner": name}})
        assert ctx.calls[-1] == want
    n = len(ctx.calls)
    api._apply_solver_config(ctx, {"solver_parameters": {}})
    api._apply_solver_config(ctx, None)
    assert len(ctx.calls) == n
    import pytest
    with pytest.raises(ValueError):
        api._apply_solver_config(ctx, {"solver_parameters": {"preconditioner": "ilu"}})
