"""The command-line driver that replaces main.cu's loop (gisspa_main <config>): reference
config syntax, LST micrograph list, Euler file, MRC template stack and micrographs, pick-list
output.  Its lines must equal, byte for byte, what the C-ABI gives for the same inputs."""
import os
import subprocess

import numpy as np
import pytest

import gisspa
import synth
from parity import SMALL, small_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(os.path.dirname(HERE), "gisspa_v2.0_b200", "_build", "gisspa_main")


def write_mrc(path, data):
    data = np.ascontiguousarray(data, dtype="<f4")
    if data.ndim == 2:
        data = data[None]
    nz, ny, nx = data.shape
    hdr = np.zeros(256, dtype="<i4")
    hdr[0], hdr[1], hdr[2], hdr[3] = nx, ny, nz, 2  # mode 2: float32
    with open(path, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(data.tobytes())


def test_cli_matches_the_c_abi(tmp_path):
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    data2 = dict(SMALL["norm_l256_w9"][0], seed=31)
    img2 = synth.make_case(**data2).image
    write_mrc(tmp_path / "templates.mrc", tmpl)
    write_mrc(tmp_path / "m0.mrc", img)
    write_mrc(tmp_path / "m1.mrc", img2)
    euler = np.array([[10.0 * i, 5.0 * i, 0.0] for i in range(tmpl.shape[0])], np.float32)
    (tmp_path / "euler.txt").write_text("".join(f"{a:f} {b:f} {c:f}\n" for a, b, c in euler))
    ctfs = [ctf, gisspa.Ctf(ctf.defocus + 0.2, ctf.dfdiff, ctf.dfang + 10.0)]
    paths = [str(tmp_path / "m0.mrc"), str(tmp_path / "m1.mrc")]
    (tmp_path / "list.lst").write_text(
        "# micrographs\n" + "".join(f"0 {p} defocus={c.defocus:f} dfdiff={c.dfdiff:f} dfang={c.dfang:f}\n"
                                    for p, c in zip(paths, ctfs)))
    keys = dict(SMALL["norm_l256_w9"][1])
    keys["Highres"], keys["Lowres"] = keys.pop("highres"), keys.pop("lowres")
    conf = "".join(f"{k} = {v}\n" for k, v in keys.items())
    conf += (f"input = {tmp_path / 'list.lst'}\ntemplate = {tmp_path / 'templates.mrc'}\n"
             f"eulerfile = {tmp_path / 'euler.txt'}\noutput = {tmp_path / 'out.lst'}\n"
             "first = 0\nlast = 2\nGPU_ID = 0\nunknown_key = ignored\n")
    (tmp_path / "search.conf").write_text(conf)
    r = subprocess.run([CLI, str(tmp_path / "search.conf")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = (tmp_path / "out.lst").read_text()

    # the same search through the C-ABI; the CLI reads ctf fields back from the LST text
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    want = []
    for p, c, im in zip(paths, ctfs, (img, img2)):
        c2 = gisspa.Ctf(float(f"{c.defocus:f}"), float(f"{c.dfdiff:f}"), float(f"{c.dfang:f}"))
        for pk in s.search(im, c2):
            j = int(pk["template_id"])
            want.append(gisspa.format_pick(pk, 0, p, c2, float(euler[j, 0]), float(euler[j, 1])))
    assert len(want) > 0
    assert got == "".join(want)


def test_cli_templates_from_volume(tmp_path):
    """template_volume: the driver projects a 3D map on the GPU at the Euler file's angles
    (degrees, converted with the reference's pi) instead of reading a template stack."""
    from fixture_data import bump_volume

    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    vol = bump_volume(64, 60, 13)
    write_mrc(tmp_path / "map.mrc", vol)
    write_mrc(tmp_path / "m0.mrc", img)
    euler = np.array([[10.5, 20.25, 30.0], [75.0, 140.5, 3.25], [120.125, 300.0, 45.5]], np.float32)
    (tmp_path / "euler.txt").write_text("".join(f"{a:f} {b:f} {c:f}\n" for a, b, c in euler))
    path = str(tmp_path / "m0.mrc")
    (tmp_path / "list.lst").write_text(f"0 {path} defocus={ctf.defocus:f} dfdiff={ctf.dfdiff:f} dfang={ctf.dfang:f}\n")
    keys = dict(SMALL["norm_l256_w9"][1])
    keys["Highres"], keys["Lowres"] = keys.pop("highres"), keys.pop("lowres")
    conf = "".join(f"{k} = {v}\n" for k, v in keys.items())
    conf += (f"input = {tmp_path / 'list.lst'}\ntemplate_volume = {tmp_path / 'map.mrc'}\n"
             f"eulerfile = {tmp_path / 'euler.txt'}\noutput = {tmp_path / 'out.lst'}\n"
             "first = 0\nlast = 1\nGPU_ID = 0\n")
    (tmp_path / "search.conf").write_text(conf)
    r = subprocess.run([CLI, str(tmp_path / "search.conf")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = (tmp_path / "out.lst").read_text()

    rad = (euler.astype(np.float64) * 3.1415926535 / 180.0).astype(np.float32)
    s = gisspa.Searcher(cfg)
    s.set_templates_from_volume(vol, rad)
    c2 = gisspa.Ctf(float(f"{ctf.defocus:f}"), float(f"{ctf.dfdiff:f}"), float(f"{ctf.dfang:f}"))
    want = [gisspa.format_pick(pk, 0, path, c2, float(euler[int(pk["template_id"]), 0]),
                               float(euler[int(pk["template_id"]), 1])) for pk in s.search(img, c2)]
    assert len(want) > 0
    assert got == "".join(want)
