"""C ABI: the library loads and exports every symbol include/*.h declares, and
the host-only entry points (options, argv parsing) behave like RegOpt.
No compute calls: runs without a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(claire_b200_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "claire_b200_run" in names and "claire_b200_interp3" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    import claire_b200
    lib = ctypes.CDLL(claire_b200.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_opts_match_regopt_initialize():
    import claire_b200 as cb
    o = cb.RegOpt().opts
    # src/RegOpt.cpp:1032-1293
    assert o.nt == 4 and tuple(o.nx) == (32, 32, 32)
    assert o.regnorm == cb.NORMS["h1s"] and o.model == cb.MODELS["relaxedstokes"]
    assert o.beta[0] == 1e-2 and o.beta[1] == 1e-4 and o.beta[2] == 1e-4
    assert o.maxit == 50 and o.opttol == 5e-2 and o.gatol == 1e-6
    assert o.krylovmaxit == 50 and o.krylovtol[0] == 1e-12 and o.krylovtol[1] == 1e-16
    assert o.krylovtol[2] == 1e6 and o.precond == 1 and o.iporder == 3


def test_parse_args():
    import claire_b200 as cb
    opt = cb.RegOpt(["-nx", "64x64x64", "-nt", "8", "-regnorm", "h2", "-beta", "1e-3", "-maxit", "10",
                     "-opttol", "1e-2", "-krylovfseq", "quadratic", "-precond", "invreg"])
    o = opt.opts
    assert tuple(o.nx) == (64, 64, 64) and o.nt == 8
    assert o.regnorm == cb.NORMS["h2"] and o.model == cb.MODELS["compressible"]
    assert o.beta[0] == 1e-3 and o.maxit == 10 and o.opttol == 1e-2 and o.krylovfseq == 1
    assert o.bf16_images == 0
    assert cb.RegOpt(["-nx", "64", "-bf16images"]).opts.bf16_images == 1
    assert o.autotune == 0 and cb.RegOpt(["-nx", "64", "-autotune"]).opts.autotune == 1
    assert o.distance == 0 and cb.RegOpt(["-nx", "64", "-distance", "ncc"]).opts.distance == 1
    assert o.train == 0 and o.jbound == 0.25 and o.betainit == 1.0
    t = cb.RegOpt(["-nx", "64", "-train", "binary", "-jbound", "0.3", "-betainit", "0.5"]).opts
    assert t.train == 1 and t.jbound == 0.3 and t.betainit == 0.5
    with pytest.raises(cb.ClaireError):
        cb.RegOpt(["-nx", "64", "-betacont", "1e-3", "-train", "reduce"])
    opt2 = cb.RegOpt(["-nx", "96", "-regnorm", "h1s-stokes"])
    assert tuple(opt2.opts.nx) == (96, 96, 96) and opt2.opts.model == cb.MODELS["stokes"]


def test_parse_args_rejects_bad_input():
    import claire_b200 as cb
    with pytest.raises(cb.ClaireError):
        cb.RegOpt(["-regnorm", "h7"])
    with pytest.raises(cb.ClaireError):
        cb.RegOpt(["-iporder", "1"])
    with pytest.raises(cb.ClaireError):
        cb.RegOpt(["-nx"])


def test_memory_estimate_scales():
    import claire_b200 as cb
    a = cb.RegOpt(["-nx", "64", "-nt", "4"]).estimate_bytes(1)
    b = cb.RegOpt(["-nx", "128", "-nt", "4"]).estimate_bytes(1)
    assert 7.5 < b / a < 8.5
    assert cb.RegOpt(["-nx", "64"]).estimate_bytes(4) == 4 * a


def test_parse_betacont():
    import claire_b200 as cb
    o = cb.RegOpt(["-nx", "32", "-betacont", "1e-4"]).opts
    assert o.betacont == 1e-4 and o.presolvetol == 1e-1
    assert cb.RegOpt().opts.betacont == 0.0


def test_parse_two_level_preconditioner():
    # src/RegOpt.cpp:592-650 and the defaults of :1120-1124
    import claire_b200 as cb
    d = cb.RegOpt().opts
    assert d.pcgridscale == 2.0 and d.pctolscale == 0.1 and d.pcsolvermaxit == 10
    o = cb.RegOpt(["-nx", "64", "-precond", "2level", "-gridscale", "4", "-pctolscale", "0.05",
                   "-pcsolvermaxit", "5", "-pcsolver", "pcg", "-monitorpcsolver"]).opts
    assert o.precond == 2 and o.pcgridscale == 4.0 and o.pctolscale == 0.05 and o.pcsolvermaxit == 5
    assert cb.RegOpt(["-precond", "none"]).opts.precond == 0
    for bad in (["-precond", "amg"], ["-pctolscale", "1.5"], ["-gridscale", "0.5"]):
        with pytest.raises(cb.ClaireError) as e:
            cb.RegOpt(bad)
        assert e.value.code == -1
    for other in ("gmres", "fgmres", "fpcg", "cheb"):
        with pytest.raises(cb.ClaireError) as e:
            cb.RegOpt(["-pcsolver", other])
        assert e.value.code == -6  # flexible / Chebyshev coarse solvers are not on this path
    # the coarse problems and the grid-change workspace are part of the footprint
    a = cb.RegOpt(["-nx", "64", "-nt", "4"]).estimate_bytes(2)
    b = cb.RegOpt(["-nx", "64", "-nt", "4", "-precond", "2level"]).estimate_bytes(2)
    assert 1.1 * a < b < 1.5 * a
