"""(CPU) The webdata file format of export_binary_for_web
(src/IO/Postprocessing.jl:239-261) as the reader sees it: a file assembled by
hand from the oracle's restated arrays parses back field by field, and the
restated centroids are the Float32 corner sums of generate_mesh's nodes."""
import struct

import numpy as np


def test_format_round_trip(hx, orc, tmp_path):
    from importlib import import_module
    api = import_module(hx.__name__ + ".api")
    dims, h = (4, 3, 2), (1.0, 1.0, 1.0)
    nodes, el, _ = hx.mesh.generate_mesh(*dims)
    n = el.shape[0]
    dens = np.linspace(0, 1, n, dtype=np.float32)
    l1 = np.ones(n, np.float32)
    pr = np.tile(np.array([1.0, -3.0, 2.0], np.float32), (n, 1))
    cent, d, s = orc.webdata_arrays(dims, h, dens, l1, pr, np.float32(0.5))
    # centroids: the mean of the element's node coordinates
    sel = np.nonzero(dens >= np.float32(0.5))[0]
    want = nodes[el[sel] - 1].mean(axis=1)
    assert np.allclose(cent, want, rtol=0, atol=1e-6)
    assert np.all(s == -1.0)  # the largest |principal| is -3
    js = b'{"iteration":3}'
    blob = struct.pack("<IIiffIfff", 0x48455841, 2, 3, 1.5, 0.5, d.size, *h)
    blob += cent.astype("<f4").tobytes() + d.astype("<f4").tobytes() + s.astype("<f4").tobytes()
    blob += struct.pack("<I", len(js)) + js
    p = tmp_path / "w.bin"
    p.write_bytes(blob)
    w = api.read_webdata(p)
    assert w["count"] == d.size and w["config"] == {"iteration": 3}
    assert np.array_equal(w["centroids"], cent) and np.array_equal(w["signed_l1"], s)
