"""The benchmark configurations at full mesh size against the reference run
on them (tests/golden/make_config_golden.py): 64^3 jittered cavity
(1,572,864 tets), 96x16x16 channel (147,456 tets) and the conjugate-heat-
transfer slab (552,960 tets), three steps each.  Time steps are bitwise; the
fields agree to RUN_TOL relative L2 at 4,000 seeded nodes and in norm."""
import json
import os
import sys

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-8
HERE = os.path.dirname(os.path.abspath(__file__))


def _load(name):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_config_golden as mk
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    g = json.loads(bytes(z["generator"]).decode())
    case = mk.build(g["gen"], g["kw"])
    assert mk.mesh_digest(case) == bytes(z["mesh_sha256"]).decode()
    return case, z


@pytest.mark.parametrize("two_level", [False, True])
@pytest.mark.parametrize("name", ["cfg2_cavity64", "cfg4_channel", "cfg5_cht"])
def test_config_full_size_vs_reference(name, two_level):
    """Jacobi (the reference's preconditioner) and the two-level extension,
    which takes fewer iterations to the same stopping test."""
    from cbs3d import gpu
    case, z = _load(name)
    n = int(z["nsteps"][0])
    hist = z["history"].reshape(n, 21)
    ctx = gpu.Context(case, two_level=two_level)
    for s in range(n):
        st = ctx.step(1)
        assert st.dtreal == hist[s, 0]
        if not two_level:
            assert abs(st.cg.iterations - int(hist[s, 1])) <= 3
    u, p, t = ctx.fields()
    idx = z["idx"]
    assert rel_l2(u.reshape(-1, 3)[idx], z["u"]) <= RUN_TOL
    assert rel_l2(p[idx], z["p"]) <= RUN_TOL
    assert abs(np.linalg.norm(u) - z["norm_u"][0]) <= RUN_TOL * z["norm_u"][0]
    assert abs(np.linalg.norm(p) - z["norm_p"][0]) <= RUN_TOL * z["norm_p"][0]
    if case.params.get("temp_calc", 0):
        assert rel_l2(t[idx], z["t"]) <= RUN_TOL
        assert abs(np.linalg.norm(t) - z["norm_t"][0]) <= RUN_TOL * z["norm_t"][0]
