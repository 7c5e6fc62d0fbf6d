"""CPU checks of the C-ABI library: it loads, exports every declared symbol, parses the
reference config format and formats pick lines; no device is needed."""
import ctypes as C
import os
import re
import sys

import numpy as np
import pytest

import gisspa

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(REPO, "include", "gisspa.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gisspa_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = gisspa.load()
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(gisspa.SIGNATURES)


def test_version():
    assert b"sm_100a" in gisspa.load().gisspa_version()


def test_config_defaults_match_reference():
    c = gisspa.Config()
    gisspa.load().gisspa_config_default(C.byref(c))
    assert c.window_size == 320 and c.threshold == pytest.approx(7.0) and c.norm_type == 0
    assert c.edge_half_width == 4.0 and c.ampconst == pytest.approx(0.07) and c.a == pytest.approx(-10.81)
    assert c.quirks == gisspa.QUIRKS_REFERENCE and c.tile_size == 720
    assert c.cuda_graphs == 1 and c.pass_b_shape == -1
    assert c.pass_a_shape == -1 and c.prune_sweep2 == 1 and c.tensor_cores == 0


def test_config_file_parsing(tmp_path):
    p = tmp_path / "config"
    p.write_text("input = mics.lst\ntemplate = t.hdf\neulerfile = e.txt\nangpix = 1.3\nphistep = 5\nkk = 3\n"
                 "energy = 300\ncs = 2.7\nHighres = 8\nLowres = 200\ndiameter = 180\nthreshold = 7.5\n"
                 "output = out.lst\nfirst = 2\nlast = 9\nGPU_ID = 1\nwindow_size = 512\nphase_flip = 1\n"
                 "overlap = 192\nnorm_type = 1\ninvert = 1\nunknown_key = whatever\npick_mode = topk\n"
                 "spectrum_precision = fp16\ntopk = 50\ncuda_graphs = 0\npass_b_shape = 2\ntemplate_batch = 24\n"
                 "window_batch = 4\npass_a_shape = 1\nprune_sweep2 = 0\n")
    c, r = gisspa.load_config(str(p))
    assert (c.angpix, c.phistep, c.window_size, c.overlap, c.norm_type, c.invert) == (
        pytest.approx(1.3), 5.0, 512, 192, 1, 1)
    assert c.pick_mode == gisspa.PICK_TOPK and c.spectrum_precision == gisspa.SPEC_FP16 and c.topk == 50
    assert (c.cuda_graphs, c.pass_b_shape, c.template_batch, c.window_batch) == (0, 2, 24, 4)
    assert (c.pass_a_shape, c.prune_sweep2) == (1, 0)
    assert r.input == b"mics.lst" and r.template_path == b"t.hdf" and (r.first, r.last, r.gpu_id) == (2, 9, 1)


def test_config_errors(tmp_path):
    with pytest.raises(gisspa.GisspaError) as e:
        gisspa.load_config(str(tmp_path / "missing"))
    assert e.value.status == gisspa.ERR_IO
    p = tmp_path / "bad"
    p.write_text("window_size = abc\n")
    with pytest.raises(gisspa.GisspaError):
        gisspa.load_config(str(p))


def test_format_pick_matches_reference_line():
    p = np.zeros(1, dtype=gisspa.PICK_DTYPE)[0]
    p["score"], p["x"], p["y"], p["angle"] = 7.25, 100.0, 200.0, 355.0
    line = gisspa.format_pick(p, 3, "mic.mrc", gisspa.Ctf(1.5, 0.1, 30.0), 12.0, 45.0)
    assert line == ("3\tmic.mrc\tdefocus=1.500000\tdfdiff=0.100000\tdfang=30.000000\teuler=12.000000,45.000000,"
                    "355.000000\tcenter=100.000000,200.000000\tscore=7.250000\n")


def test_create_rejects_bad_configs():
    lib = gisspa.load()
    h = C.c_void_p()
    for over in [dict(window_size=300), dict(window_size=16), dict(window_size=4096), dict(phistep=0.0),
                 dict(overlap=600),
                 dict(pass_b_shape=9), dict(pass_b_shape=-2), dict(pass_a_shape=2), dict(pass_a_shape=-2)]:
        cfg = gisspa.Config.default(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                                    lowres=200.0, diameter=100.0, window_size=512, norm_type=1, **{})
        for k, v in over.items():
            setattr(cfg, k, v)
        st = lib.gisspa_create(C.byref(cfg), 0, C.byref(h))
        assert st in (gisspa.ERR_SHAPE, gisspa.ERR_UNSUPPORTED, gisspa.ERR_ARG), (over, st)
        assert lib.gisspa_last_error(None)


def test_null_handle_is_an_argument_error():
    lib = gisspa.load()
    n = C.c_size_t(0)
    assert lib.gisspa_search(None, None, 0, 0, None, None, 0, C.byref(n)) == gisspa.ERR_ARG
    assert lib.gisspa_set_templates(None, None, 0, 0, 0) == gisspa.ERR_ARG


def test_null_handle_new_entry_points():
    lib = gisspa.load()
    n = C.c_size_t(0)
    assert lib.gisspa_shard_sweep(None, 1, 0, 1) == gisspa.ERR_ARG
    assert lib.gisspa_shard_export(None, None, None, None) == gisspa.ERR_ARG
    assert lib.gisspa_shard_picks(None, None, 0, C.byref(n)) == gisspa.ERR_ARG
    assert lib.gisspa_debug_wait_probe(None, 0.1) == gisspa.ERR_ARG


def test_timing_script_writes_configs_the_reference_syntax_reads(tmp_path):
    """oracle/ref_time.py hands the same config files to the reference build and to
    gisspa_main: the library's parser (the reference's key syntax) reads back the workload."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_time
    import synth

    wl = "whole_2048_t24"
    d = str(tmp_path)
    lst1, lst2 = ref_time.write_inputs(d, wl)
    cfgp = os.path.join(d, "config")
    ref_time.write_config(cfgp, wl, d, lst2, 2, os.path.join(d, "picks.txt"))
    c, r = gisspa.load_config(cfgp)
    want = synth.SEARCH_PARAMS[wl]
    assert (c.window_size, c.overlap, c.norm_type) == (want["window_size"], want["overlap"], want["norm_type"])
    assert (c.phistep, c.highres, c.lowres, c.diameter) == (want["phistep"], want["highres"], want["lowres"],
                                                            want["diameter"])
    assert (r.first, r.last, r.gpu_id) == (0, 2, 0) and r.input.decode() == lst2
    with open(lst2) as fh:
        assert sum(1 for ln in fh if ln.strip() and not ln.startswith("#")) == 2
