"""Boundary-condition and load mapping of src/Core/Boundary.jl (host side).

Restates the location grammar (Boundary.jl:56-130): a component is ":" (all),
a number in [0, 1] read as a FRACTION of the bounding box, any other number
read as an absolute coordinate, or a "P%" string; nodes within
1e-4*max(1, extent) of the value match.  Forces given by location are spread
evenly over the matched nodes (Boundary.jl:280); a point location that
matches nothing maps to the nearest node (Boundary.jl:244-260).
"""
import numpy as np


def _resolve(spec, cmin, cmax):
    """resolve_coordinate_value, Boundary.jl:109-122."""
    if isinstance(spec, str) and spec.endswith("%"):
        frac = min(max(float(spec[:-1]) / 100.0, 0.0), 1.0)
        return np.float32(cmin + frac * (cmax - cmin))
    spec = float(spec)
    if 0.0 <= spec <= 1.0:
        return np.float32(cmin + spec * (cmax - cmin))
    return np.float32(spec)


def _component_mask(spec, coords):
    """interpret_location_component, Boundary.jl:81-107."""
    cmin, cmax = coords.min(), coords.max()
    tol = np.float32(1e-4) * max(np.float32(1.0), abs(cmax - cmin))
    if isinstance(spec, str) and spec == ":":
        return np.ones(coords.shape[0], bool)
    if isinstance(spec, (int, float, np.integer, np.floating)) or (
            isinstance(spec, str) and spec.endswith("%")):
        val = _resolve(spec, cmin, cmax)
        return np.abs(coords - val) <= tol
    raise ValueError(f"Invalid location component: {spec}")


def nodes_by_location(loc, nodes):
    """get_nodes_by_location, Boundary.jl:63-79: 0-based matching node ids."""
    if len(loc) < 3:
        raise ValueError("Location specification must have at least 3 components (x,y,z)")
    m = np.ones(nodes.shape[0], bool)
    for d in range(3):
        m &= _component_mask(loc[d], nodes[:, d])
    return np.nonzero(m)[0]


def affected_nodes(spec, nodes):
    """get_affected_nodes, Boundary.jl:20-54 (0-based ids)."""
    nn = nodes.shape[0]
    if "node" in spec:
        raw = spec["node"]
        if isinstance(raw, (int, np.integer)):
            return np.array([min(max(int(raw), 1), nn) - 1])
        return np.unique([min(max(int(r), 1), nn) - 1 for r in raw])
    if "location" in spec:
        return nodes_by_location(spec["location"], nodes)
    raise ValueError("Specification must include either 'node' or 'location'")


def get_bc_indicator(n_nodes, nodes, bc_data):
    """get_bc_indicator, Boundary.jl:135-160: (nN, 3) float32, 1 = fixed."""
    bc = np.zeros((n_nodes, 3), np.float32)
    for spec in bc_data:
        dofs = spec["DoFs"]
        for d in dofs:
            if d < 1 or d > 3:
                raise ValueError(f"Invalid DoF index: {d} (must be 1..3).")
        nd = affected_nodes(spec, nodes)
        for d in dofs:
            bc[nd, d - 1] = 1.0
    return bc


def find_nearest_node(target, nodes):
    """find_nearest_node, Boundary.jl:189-222 (ties -> larger x, then y, z)."""
    d2 = ((nodes.astype(np.float64) - np.asarray(target, np.float64)) ** 2).sum(1)
    best = d2.min()
    cand = np.nonzero(np.abs(d2 - best) <= 1e-9)[0]
    order = np.lexsort((nodes[cand, 2], nodes[cand, 1], nodes[cand, 0]))
    return int(cand[order[-1]])


def apply_external_forces(F, forces_data, nodes):
    """apply_external_forces!, Boundary.jl:232-291 (F is modified and returned)."""
    for force in forces_data:
        nd = affected_nodes(force, nodes)
        if len(nd) == 0 and "location" in force:
            loc = force["location"]
            if all(not (isinstance(c, str) and c == ":") for c in loc):
                target = [_resolve(loc[d], nodes[:, d].min(), nodes[:, d].max()) for d in range(3)]
                nd = np.array([find_nearest_node(target, nodes)])
        if len(nd) == 0:
            continue
        f = np.zeros(3, F.dtype)
        raw = list(force["F"])[:3]
        f[:len(raw)] = raw
        scale = F.dtype.type(1.0) / len(nd) if "location" in force else F.dtype.type(1.0)
        for d in range(3):
            F[3 * nd + d] += scale * f[d]
    return F
