"""The key = value parameter system: syntax, aliases, booleans, errors and the
file-then-override order of src/utils/params.cpp:37-114, checked against the
reference's own parser where it was built (oracle/_ref)."""
import pytest

from lbm_solver_3d_b200.params import ParamError, Params


def test_file_syntax_comments_and_overrides(tmp_path):
    deck = tmp_path / "deck.in"
    deck.write_text("# comment line\n nx = 40  # trailing\n\nWALLS_Z = yes\nsq = on\nR=5.5\nbeta=-2\n")
    p = Params.from_args(deck, "nx=48", "beta=1.5")
    assert (p.NX, p.wallsZ, p.squirmer, p.R, p.beta) == (48, True, True, 5.5, 1.5)


@pytest.mark.parametrize("alias,attr,text,val", [
    ("walls_y", "wallsY", "off", False), ("wallsy", "wallsY", "No", False), ("print", "printEvery", "7", 7),
    ("vtk", "vtkEvery", "3", 3), ("traj", "trajEvery", "9", 9), ("sq", "squirmer", "TRUE", True),
    ("r", "R", "3", 3.0), ("rhop", "rhoP", "2", 2.0), ("rho_p", "rhoP", "2", 2.0)])
def test_aliases(alias, attr, text, val):
    p = Params()
    p.set(alias, text)
    assert getattr(p, attr) == val


def test_errors(tmp_path):
    with pytest.raises(ParamError, match="unknown parameter 'bogus'"):
        Params().set("bogus", "1")
    with pytest.raises(ParamError, match="cannot interpret 'maybe' as a boolean"):
        Params().set("planar", "maybe")
    with pytest.raises(ParamError, match="invalid value 'abc' for parameter 'nx'"):
        Params().set("nx", "abc")
    bad = tmp_path / "bad.in"
    bad.write_text("nx = 4\nthis line has no equals\n")
    with pytest.raises(ParamError, match=r"bad.in:2: expected 'key = value'"):
        Params().load_file(bad)
    with pytest.raises(ParamError, match="cannot open input file"):
        Params().load_file(tmp_path / "missing.in")


def test_stoi_stod_prefix_semantics():
    p = Params()
    p.set("nx", " 12abc")
    p.set("tau", "0.75xyz")
    assert p.NX == 12 and p.tau == 0.75


def test_extra_keys():
    p = Params().update(precision="fp32", ex=0.0, ey=1.0, ez=0.0)
    assert p.precision == "fp32" and p.orientation == (0.0, 1.0, 0.0)
    with pytest.raises(ParamError, match="precision must be one of"):
        Params().set("precision", "fp8")
    q = Params().update(checkpoint_every=500, restart="run_checkpoint.bin")
    assert q.checkpoint_every == 500 and q.restart == "run_checkpoint.bin"


def test_reference_parser_agrees(oracle_mod):
    """The reference's own Params (compiled into oracle/_ref) accepts what the
    mirror accepts and rejects what it rejects, with the same message."""
    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built")
    good = Params().update(nx=20, ny=20, nz=20, squirmer=1, radius=3, walls_y=0)
    s = oracle_mod.RefSolver(good)
    assert s.N == 8000
    for kw, msg in [(dict(tau=0.5), "tau must be > 0.5"),
                    (dict(squirmer=1, nx=9), "domain too small for the squirmer")]:
        p = Params().update(**kw)
        with pytest.raises(ParamError, match=msg):
            p.validate()
        with pytest.raises(RuntimeError, match=msg):
            oracle_mod.RefSolver(p)
