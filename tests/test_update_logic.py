"""(CPU) The oracle's restatement of update_density! (oracle.update_density,
src/Optimization/TopOpt.jl:139-405) on hand-checked cases: the radius
schedule and its guard, and the culling cap with ties culled in element
order (Julia's stable sort)."""
import numpy as np


def test_radius_schedule(orc):
    # iter 1: R = R_init = 8% of 60 = 4.8 (above the 1.2 h guard); R_eff = R / 2.5
    R, Re = orc.radius_schedule(1, 40, (1, 1, 1), 60.0, 8.0, 5.0, 3.0)
    assert abs(R - 4.8) < 1e-6 and abs(Re - R / 2.5) < 1e-15
    # at iter_interm (20 = 50% of 40) the intermediate radius; at the end the final one
    R, _ = orc.radius_schedule(20, 40, (1, 1, 1), 60.0, 8.0, 5.0, 3.0)
    assert abs(R - 3.0) < 1e-6
    R, _ = orc.radius_schedule(40, 40, (1, 1, 1), 60.0, 8.0, 5.0, 3.0)
    assert abs(R - 1.8) < 1e-6
    # below the guard 1.2 * mean h the guard applies (Float32 quotient by 2.5)
    R, Re = orc.radius_schedule(5, 40, (1, 2, 3), 60.0, 0.0, 0.0, 0.0)
    assert R == float(np.float32(1.2) * np.float32(2.0)) and Re == float(np.float32(R) / np.float32(2.5))


def test_culling_cap_and_ties(orc):
    dims = (4, 3, 2)
    n = 24
    dens = np.full(n, 0.5, np.float32)
    l1 = np.zeros(n, np.float32)
    prot = np.zeros(n, bool)
    orig = dens.copy()
    # a filtered field with runs of equal values: 0.1 (x6), 0.2 (x10), 0.9 (x8)
    filt = np.array([0.2] * 5 + [0.1] * 3 + [0.9] * 8 + [0.2] * 5 + [0.1] * 3, np.float32)
    d, _, (mc, R, thr, _, _), _ = orc.update_density(
        dens, l1, prot, 1.0, 1.0, 10, 10, orig, 1e-3, 1.0, dims, (1, 1, 1), 4.0,
        max_culling_ratio=0.5, filtered=filt)
    # active 24, cap floor(24 * 0.5) = 12 of 16 candidates (< 0.95): the six
    # 0.1 values, then the first six 0.2 values in element order
    culled = np.nonzero(d == np.float32(1e-3))[0]
    assert list(culled) == [0, 1, 2, 3, 4, 5, 6, 7, 16, 21, 22, 23]
    f32 = np.float32
    assert thr == float(f32(0.95) * (f32(10) / f32(10)))
    assert mc == float(max(f32(0.5) - f32(0.1), f32(0.9) - f32(0.5)))
