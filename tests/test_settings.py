import json

import pytest

from zoomy_dmplex_b200 import native
from zoomy_dmplex_b200.settings import Settings, SolverSettings


def test_from_json_defaults_and_mapping(tmp_path):
    p = tmp_path / "s.json"
    p.write_text(json.dumps({"name": "x", "solver": {"cfl": 0.45, "reconstruction_order": 2, "ssp_stages": 2,
                                                       "limiter": "venkatakrishnan"},
                             "model": {"parameters": {"g": 9.8, "n_manning": 0.03, "bogus": "s"}}}))
    s = Settings.from_json(str(p))
    assert s.solver.cfl == 0.45 and s.solver.ssp_stages == 2 and s.solver.min_dt == 1e-12
    st = s.solver.to_struct()
    # any limiter other than "none" installs vacuum + TVD (Reconstruction.hpp:170-175)
    assert st.limiter == native.ZSME_LIMITER_TVD
    # Green-Gauss is what the reference's MUSCL path installs (ModularSolver.hpp:62-67)
    assert st.gradient == native.ZSME_GRADIENT_GREEN_GAUSS
    assert SolverSettings(gradient="least_squares").to_struct().gradient == native.ZSME_GRADIENT_LSQ
    assert s.parameters == {"g": 9.8, "n_manning": 0.03}
    assert SolverSettings(limiter="none").to_struct().limiter == native.ZSME_LIMITER_NONE
    assert SolverSettings().ssp_stages == 5          # reference default


def test_rejects_out_of_path_strategies():
    with pytest.raises(ValueError):
        SolverSettings(time_integration="explicit_only").to_struct()
    assert SolverSettings(time_integration="imex").to_struct().time_integration == native.ZSME_TIME_IMEX
    assert SolverSettings(time_integration="implicit").to_struct().time_integration == native.ZSME_TIME_IMPLICIT
    assert SolverSettings().to_struct().refresh_derivative_aux == 1     # the reference's default
    with pytest.raises(ValueError):
        SolverSettings(positivity="bogus").to_struct()
    assert SolverSettings(positivity="mood").to_struct().positivity == native.ZSME_POSITIVITY_MOOD
    st = SolverSettings(positivity="zhang_shu", wet_dry_eps=0.05).to_struct()
    assert st.positivity == native.ZSME_POSITIVITY_ZHANG_SHU and st.wet_dry_eps == 0.05
