"""Declarative scene specs (octopusengine_b200/spec.py): names map onto the reference's enums
and the benchmark configurations build the meshes the configs describe."""
import json

import numpy as np
import pytest

import oracle_lib as O


def test_config_specs_build_the_configured_meshes(built):
    from octopusengine_b200 import spec
    e, X, T, kw = spec.mesh_and_kwargs(spec.load("config1"))
    assert e == O.TETRA and len(X) == 81 and len(T) == 192
    assert kw["young"] == 1e5 and kw["iterations"] == 20 and len(kw["fixed_ids"]) == 9
    e, X, T, kw = spec.mesh_and_kwargs(spec.load("config2"))
    assert e == O.TETRA10 and len(X) == 129 * 33 * 33 and len(T) == 98304
    assert kw["initial_velocity"].shape == X.shape and abs(kw["initial_velocity"].std() - 0.05) < 1e-3


def test_json_round_trip_and_enum_names(built, tmp_path):
    from octopusengine_b200 import capi, spec
    s = dict(spec.CONFIGS["config1"], material="Hooke", solver="XPBD", xpbd_version="Quadrature", precision="mixed")
    path = tmp_path / "scene.json"
    path.write_text(json.dumps(s))
    e, X, T, kw = spec.mesh_and_kwargs(spec.load(str(path)))
    assert kw["material"] == capi.HOOKE and kw["solver"] == capi.SOLVER_XPBD
    assert kw["xpbd_version"] == capi.XPBD_QUADRATURE and kw["precision"] == capi.PREC_MIXED
    with pytest.raises(ValueError):
        spec.mesh_and_kwargs(dict(s, material="Rubber"))


@pytest.mark.gpu
def test_config1_spec_steps_like_the_oracle(ctx):
    from octopusengine_b200 import spec
    from scenes import rel_err
    sc, dt, sub = spec.scene(ctx, spec.load("config1"))
    e, X, T, kw = spec.mesh_and_kwargs(spec.load("config1"))
    m = O.masses(e, X, T, 1000.0, 1)
    c, n = O.colour(e, T, len(X), 0)
    ref = O.Solver("vbd", O.Scene(e, X, T, m, young=1e5, fixed=kw["fixed_ids"], iterations=20, colors=c, n_colors=n,
                                  in_place=True), fp64=True)
    for _ in range(3):
        sc.step(dt, sub)
        ref.step(dt, sub)
    assert rel_err(sc.get_position(), ref.get(0)) < 1e-5
