"""The full-size fixtures (tests/golden/full_*.npz) on the CPU: their seeds
regenerate exactly the catalogues they were made from (the digest each
fixture recorded), and the unit-weight fixtures hold integer counts."""
import os

import numpy as np
import pytest

from two_pcf_b200 import synthetic

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = [n for n in ("full_box", "full_survey_unit", "full_survey_w")
         if os.path.exists(os.path.join(HERE, "golden", n + ".npz"))]


@pytest.mark.parametrize("name", NAMES)
def test_fixture_inputs_regenerate(name):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    if name == "full_box":
        w = synthetic.box_catalogue(seed=int(g["gen_seed"]), n_data=int(g["gen_n_data"]),
                                    n_rand=int(g["gen_n_rand"]))
        d, r = {"xyz": w["data"]["xyz"]}, {"xyz": w["rand"]["xyz"]}
    else:
        w = synthetic.survey_catalogue(seed=int(g["gen_seed"]), n_data=int(g["gen_n_data"]),
                                       n_rand=int(g["gen_n_rand"]))
        d, r = w["data"], w["rand"]
        if name == "full_survey_unit":
            for c in (d, r):
                c["weight"] = np.ones_like(c["weight"])
    assert synthetic.catalogue_digest(d) == str(g["digest_data"])
    assert synthetic.catalogue_digest(r) == str(g["digest_rand"])
    if name != "full_survey_w":
        for k in g.files:
            if k.endswith(("_full", "_sub")) and not k.startswith("xi") and "_norm_" not in k and "_xi_" not in k:
                v = g[k]
                assert np.array_equal(v, np.round(v)), k
