"""The model-input loader (tissueorigami_b200.modelinput) on the reference's own input.

The Pardiso regression run 07008 of the reference recorded the set-up it derived from its
model input - Young's modulus per element, external viscosity per node, the binding pairs, the
ECM elements - and its first step's positions (tests/golden/run07008_newton_step1.npz, with the
model input file's tokens). The loader must derive the same set-up from the same model input
and mesh by the reference's rules, and that set-up must give the recorded first step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import modelinput as MI

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run07008_newton_step1.npz")


def _load():
    z = np.load(GOLDEN)
    text = " ".join(str(t) for t in z["modelinput_tokens"])
    st = MI.setup(MI.parse(text), (z["x"], z["place"], z["ttype"], z["circ"], z["conn"], z["xref"]))
    return st, z


def test_parse_keeps_keys_values_and_order():
    e = MI.parse("Sec:\n  A(x): 1 2 3  B: 4\nGrowthFunctionType(int): 1\n  Angle(degrees): 45\n"
                 "GrowthFunctionType(int): 3\n")
    assert e == [("Sec", []), ("A(x)", ["1", "2", "3"]), ("B", ["4"]), ("GrowthFunctionType(int)", ["1"]),
                 ("Angle(degrees)", ["45"]), ("GrowthFunctionType(int)", ["3"])]


def test_setup_matches_what_the_reference_recorded():
    st, z = _load()
    t = st.tissue
    nu = np.where(st.ecm, 0.0, 0.29)
    np.testing.assert_array_equal(st.ecm, z["ecm"])
    np.testing.assert_allclose(2 * t.mu * (1 + nu), z["young"], rtol=1e-15)
    np.testing.assert_array_equal(t.eta, z["eta"])
    np.testing.assert_array_equal(t.ext_visc, z["ext_visc"])
    np.testing.assert_array_equal(t.fixed, z["fixed"])
    np.testing.assert_array_equal(t.exposed, z["exposed"])
    assert sorted(map(tuple, t.slave_master)) == sorted(map(tuple, z["pairs"]))
    rates, angles = st.growth_at(0.0)
    np.testing.assert_array_equal(np.any(rates != 0, axis=1), z["grown"])
    np.testing.assert_array_equal(rates[z["grown"]], np.tile(z["rates"], (int(z["grown"].sum()), 1)))
    assert (angles[z["grown"]] == float(z["angle"])).all()
    assert not st.growth_at(18000.0)[0].any()  # FinalTime 18000 s
    assert t.dt == 3600.0
    assert set(st.not_modelled) == {"explicit-ECM remodelling", "adhesion", "node collapse"}


def test_unsupported_options_are_refused():
    st, z = _load()
    text = " ".join(str(t) for t in z["modelinput_tokens"]).replace("symmetricInX(bool): 0", "symmetricInX(bool): 1")
    with pytest.raises(NotImplementedError, match="symmetry"):
        MI.setup(MI.parse(text), (z["x"], z["place"], z["ttype"], z["circ"], z["conn"], z["xref"]))


def test_loaded_input_gives_the_recorded_first_step_on_the_oracle():
    st, z = _load()
    t = st.tissue.copy()
    t.rates, t.angles = st.growth_at(0.0)
    x, fg, its, norms = O.simulate_dense(t, n_steps=1)
    assert np.abs(x - z["x_step1"]).max() <= 1e-8
    assert its[0] == len(z["du_trace"])


@pytest.mark.gpu
def test_loaded_input_gives_the_recorded_first_step_on_the_gpu():
    st, z = _load()
    xs, stats = st.simulate(n_steps=1)
    assert stats[0]["rc"] == 0
    assert np.abs(xs[0] - z["x_step1"]).max() <= 1e-8
    assert stats[0]["newton_iters"] == len(z["du_trace"])


def test_save_frame_writer_reproduces_the_reference_file():
    """Writing the recorded first frame back gives the reference's Save_Frame text byte for byte."""
    from tissueorigami_b200 import mesh

    st, z = _load()
    text = str(z["frame_text"])
    (time_s, x, flags, conn), = mesh.read_save_frame(text, is_text=True)
    assert time_s == 3600.0
    np.testing.assert_array_equal(conn, z["conn"])
    np.testing.assert_array_equal(x, z["x_step1"])
    block = mesh.save_frame_block(time_s, x, flags[:, 0], flags[:, 1], flags[:, 2], conn, z["xref"])
    assert block == text


def test_save_frame_round_trip(tmp_path):
    from tissueorigami_b200 import mesh

    st, z = _load()
    t = st.tissue
    p = tmp_path / "Save_Frame"
    frames = [(3600.0, z["x_step1"]), (7200.0, z["x_step1"] + 1e-3)]
    mesh.write_save_frame(str(p), frames, t)
    back = mesh.read_save_frame(str(p))
    assert [f[0] for f in back] == [3600.0, 7200.0]
    for (tm, x), (tb, xb, flags, conn) in zip(frames, back):
        assert np.abs(xb - x).max() <= 1e-9 * np.abs(x).max()  # 10 significant digits
        np.testing.assert_array_equal(flags[:, 2], t.at_circumference)
