"""The reference's own test cases, run against the b200 mirror.

Each test restates one case of the reference's test suite
(tests/test_hit_run_metadata_and_hyperviscosity.py,
tests/test_riemann_config3_08.py, tests/test_riemann_config6.py) for the
b200 backend.  The only deliberate difference: the mirror's configs default
to backend "b200" where the reference's default to "cupy".
"""

import json
import math

import numpy as np
import pytest
import torch

from hit_solver_b200.domain import Domain2D
from hit_solver_b200.equations import EulerEquation2D
from hit_solver_b200.hit2d import HIT2DConfig, save_run_config
from hit_solver_b200.problems.riemann import (RiemannConfig3, RiemannConfig3Offset08,
                                              RiemannConfig6, hyperviscosity_enabled_for_config)


# ---- test_hit_run_metadata_and_hyperviscosity.py:22-42 ------------------------------
def test_config_json_records_resolved_configuration_and_policy(tmp_path):
    config = HIT2DConfig(nx=32, ny=24, target_mach=0.25, output_dir=tmp_path)
    path = save_run_config(tmp_path, config)
    payload = json.loads(path.read_text())
    assert path == tmp_path / "config.json"
    assert payload["nx"] == 32 and payload["ny"] == 24 and payload["target_mach"] == 0.25
    assert payload["output_dir"] == str(tmp_path)
    assert payload["problem"] == "hit2d"
    assert payload["forcing_type"] == "solenoidal_shell_ou"
    assert payload["spatial_discretization"] == "hybrid_compact_weno7"
    assert payload["hyperviscosity_policy"] == "compact_nodes_only"


# ---- test_hit_run_metadata_and_hyperviscosity.py:45-81 ------------------------------
@pytest.mark.gpu
def test_hyperviscosity_updates_only_compact_nodes():
    from hit_solver_b200.spatial_operator import PeriodicHyperviscosity2D

    domain = Domain2D(0.0, 2.0 * math.pi, 0.0, 2.0 * math.pi, 12, 10)
    equation = EulerEquation2D(gamma=1.4)
    x, y = domain.mesh()
    rho = 1.0 + 0.01 * np.sin(x) * np.cos(y)
    u = 0.02 * np.sin(y)
    v = 0.02 * np.cos(x)
    p = np.full_like(rho, 1.0 / 1.4)
    q = np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
    qd = torch.from_numpy(q).cuda()
    mask = np.zeros((domain.ny, domain.nx), dtype=bool)
    mask[3:7, 4:9] = True
    filt = PeriodicHyperviscosity2D(domain, mn=0.002)
    out = filt.apply(qd.clone(), equation, active_mask=torch.from_numpy(mask).cuda())
    diff = (out - qd).cpu().numpy()
    assert np.any(np.abs(diff[:, mask]) > 0.0)
    assert np.allclose(diff[:, ~mask], 0.0)
    with pytest.raises(ValueError):
        filt.apply(qd.clone(), equation)


# ---- test_hit_run_metadata_and_hyperviscosity.py:84-89 ------------------------------
def test_weno_only_riemann_disables_hyperviscosity():
    assert hyperviscosity_enabled_for_config(RiemannConfig3(scheme="hybrid", mn=0.001,
                                                            hyperviscosity_interval=1))
    assert not hyperviscosity_enabled_for_config(RiemannConfig3(scheme="weno", mn=0.001,
                                                                hyperviscosity_interval=1))


# ---- test_riemann_config3_08.py:12-48 ------------------------------------------------
def test_offset08_defaults():
    c = RiemannConfig3Offset08()
    assert (c.x_split, c.y_split, c.tfinal, c.cfl) == (0.8, 0.8, 0.3, 0.4)
    assert c.backend == "b200"
    assert (c.scheme, c.mn, c.hyperviscosity_interval) == ("hybrid", 0.001, 5)
    centered = RiemannConfig3()
    assert (centered.x_split, centered.y_split, centered.cfl) == (0.5, 0.5, 0.4)


@pytest.mark.gpu
def test_offset08_quadrants_are_split_at_point_eight():
    c = RiemannConfig3Offset08(nx=10, ny=10)
    q = c.initial_state()
    rho, u, v, p = (t.cpu().numpy() for t in c.equation.primitive_from_conservative(q))
    for (j, i), want in {(0, 0): (0.138, 1.206, 1.206, 0.029), (0, 9): (0.5323, 0.0, 1.206, 0.3),
                         (9, 0): (0.5323, 1.206, 0.0, 0.3), (9, 9): (1.5, 0.0, 0.0, 1.5)}.items():
        np.testing.assert_allclose((rho[j, i], u[j, i], v[j, i], p[j, i]), want, rtol=0.0, atol=1e-14)
    assert np.count_nonzero(rho == 0.138) == 64
    assert np.count_nonzero(rho == 0.5323) == 32
    assert np.count_nonzero(rho == 1.5) == 4


# ---- test_riemann_config6.py:11-49 ----------------------------------------------------
@pytest.mark.gpu
def test_config6_quadrant_states():
    c = RiemannConfig6(nx=4, ny=4)
    rho, u, v, p = (t.cpu().numpy() for t in c.equation.primitive_from_conservative(c.initial_state()))
    np.testing.assert_array_equal(rho, [[1, 1, 3, 3], [1, 1, 3, 3], [2, 2, 1, 1], [2, 2, 1, 1]])
    np.testing.assert_array_equal(u, [[-0.75] * 4, [-0.75] * 4, [0.75] * 4, [0.75] * 4])
    np.testing.assert_array_equal(v, [[0.5, 0.5, -0.5, -0.5]] * 4)
    np.testing.assert_array_equal(p, np.ones((4, 4)))


def test_config6_defaults():
    c = RiemannConfig6()
    assert c.configuration_number == 6
    assert (c.tfinal, c.cfl) == (0.25, 0.4)
    assert c.backend == "b200"
