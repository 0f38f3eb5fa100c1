"""Command-line drop-ins and outputs on the GPU: fvb_up7 (fv_up7's CLI,
composite PPM frames, raw .bin frames, frame 99 on blow-up) and fvb_keep
(keep_fv's CLI, 2-panel PNG), the device-side frame fields, and exact
checkpoint / resume."""
from __future__ import annotations

import struct
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

import fvstuff_b200 as F
from cases import riemann4

pytestmark = pytest.mark.gpu
BIN = Path(F.__file__).resolve().parent / "bin"


def _ppm(path):
    data = path.read_bytes()
    parts = data.split(b"\n", 3)
    assert parts[0] == b"P6" and parts[2] == b"255"
    w, h = map(int, parts[1].split())
    assert len(parts[3]) == 3 * w * h
    return w, h, np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


def _png(path):
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        ln, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + ln]
        crc, = struct.unpack(">I", data[pos + 8 + ln:pos + 12 + ln])
        assert crc == zlib.crc32(typ + body) & 0xFFFFFFFF
        if typ == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        if typ == b"IDAT":
            idat += body
        pos += 12 + ln
    raw = zlib.decompress(idat)
    assert len(raw) == h * (3 * w + 1)
    return w, h


def test_fvb_up7_d2av_frames(tmp_path):
    """--d2av: the .bak's positional arguments (N C2 Cg sc order) and its
    composite; the state written at the end equals a library run"""
    r = subprocess.run([str(BIN / "fvb_up7"), "--d2av", "48", "0.6", "0.01", "0.05", "3", "--t-end", "0.02",
                        "--frames", "2", "--save", "end.ckpt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert "C2=0.600" in r.stdout and "order=3" in r.stdout and "frame  2/2" in r.stdout
    for k in range(3):
        w, h, img = _ppm(tmp_path / ("sod_%04d.ppm" % k))
        assert (w, h) == (96, 96)
    s = F.Solver(48, order=3, flux="up_hllc_d2av")
    s.set_d2av(0.6, 0.01, 0.05)
    s.init_case("sod", rho_in=10.0)
    s.advance(0.01)
    s.advance(0.02)
    want = s.get_state(layout="cons", interior=True)
    c = F.Solver(48, order=3, flux="up_hllc_d2av")
    c.load(str(tmp_path / "end.ckpt"))
    assert abs(c.sync().t - 0.02) < 1e-15
    assert np.array_equal(c.get_state(layout="cons", interior=True), want)


@pytest.mark.parametrize("args,order,flux", [(["--order", "9"], 9, "up_ducros"),
                                               (["--d2av", "40", "0.5", "0", "0.05", "9"], 9, "up_hllc_d2av")])
def test_fvb_up7_order9(tmp_path, args, order, flux):
    """UP9 from the command line: fv_up7 built with ORDER 9, and the .bak's
    fifth argument 9; the state at the end equals a library run"""
    if args[0] == "--order":
        args = ["40"] + args
    r = subprocess.run([str(BIN / "fvb_up7"), *args, "--t-end", "0.01", "--frames", "1", "--save", "end.ckpt"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "order=9" in r.stdout and "UP9" in r.stdout
    s = F.Solver(40, order=order, flux=flux)
    if flux == "up_hllc_d2av":
        s.init_case("sod", rho_in=10.0)
    else:
        s.init_case("sod")
    s.advance(0.01)
    c = F.Solver(40, order=order, flux=flux)
    c.load(str(tmp_path / "end.ckpt"))
    assert np.array_equal(c.get_state(layout="cons", interior=True), s.get_state(layout="cons", interior=True))


def test_fvb_up7_metrics_lines(tmp_path):
    """--metrics: one JSON line per frame and one at the end, with the step,
    time and throughput of the run"""
    import json
    r = subprocess.run([str(BIN / "fvb_up7"), "64", "--t-end", "0.02", "--frames", "2", "--no-ppm", "--metrics",
                        "m.jsonl"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in (tmp_path / "m.jsonl").read_text().splitlines()]
    assert [x["event"] for x in lines] == ["frame", "frame", "done"]
    assert lines[0]["t"] == pytest.approx(0.01, abs=1e-15) and lines[-1]["t"] == pytest.approx(0.02, abs=1e-15)
    assert lines[0]["step"] < lines[1]["step"] == lines[2]["step"]
    assert all(x["n"] == 64 and x["precision"] == "f64" and x["cell_stage_per_s"] > 0 for x in lines)
    assert lines[-1]["hbm_gbs"] == pytest.approx(lines[-1]["cell_stage_per_s"] * 256 / 3 / 1e9, rel=1e-5)


def test_fvb_up7_frames(tmp_path):
    r = subprocess.run([str(BIN / "fvb_up7"), "48", "--t-end", "0.02", "--frames", "2", "--bin"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "Done:" in r.stdout and "frame  2/2" in r.stdout
    for k in range(3):
        w, h, img = _ppm(tmp_path / ("sod_%04d.ppm" % k))
        assert (w, h) == (96, 96)
        raw = (tmp_path / ("sod_%04d.bin" % k)).read_bytes()
        n, = struct.unpack("<i", raw[:4])
        assert n == 48 and len(raw) == 4 + 2 * 4 * n * n
        rho = np.frombuffer(raw[4:4 + 4 * n * n], np.float32).reshape(n, n)
        assert 0.1 < rho.min() and rho.max() < 11.5
    # the density panel of the initial frame is symmetric under y -> -y
    # (circular Sod), to within one colour level
    _, _, img0 = _ppm(tmp_path / "sod_0000.ppm")
    panel = img0[:48, :48].astype(int)
    assert np.max(np.abs(panel - panel[::-1, :])) <= 1


def test_fvb_up7_resume_matches_straight_run(tmp_path):
    args = [str(BIN / "fvb_up7"), "32", "--case", "vortex", "--t-end", "0.4", "--frames", "2", "--no-ppm", "--bin"]
    subprocess.run(args + ["--save", "full.ckpt"], cwd=tmp_path, check=True, capture_output=True, timeout=120)
    half = [str(BIN / "fvb_up7"), "32", "--case", "vortex", "--t-end", "0.2", "--frames", "1", "--no-ppm",
            "--save", "half.ckpt"]
    subprocess.run(half, cwd=tmp_path, check=True, capture_output=True, timeout=120)
    s1 = F.Solver(32, bc="periodic", x0=-5, y0=-5, length=10.0)
    s1.load(tmp_path / "full.ckpt")
    s2 = F.Solver(32, bc="periodic", x0=-5, y0=-5, length=10.0)
    s2.load(tmp_path / "half.ckpt")
    assert s2.sync().t == pytest.approx(0.2, abs=1e-15)
    s2.advance(0.4)
    assert s2.sync().t == s1.sync().t
    # frame-clamped stepping differs between the two runs only in where the
    # stops fall; both land on 0.4 through the same schedule of stops here
    assert np.array_equal(s1.get_state(), s2.get_state())


@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_checkpoint_resume_is_exact(tmp_path, prec):
    n = 40
    a = F.Solver(n, bc="transmissive", precision=prec, cfl=0.5)
    a.set_state(riemann4(n, seed=3), interior=True)
    a.step(7)
    a.save(tmp_path / "c.ckpt")
    a.step(9)
    b = F.Solver(n, bc="transmissive", precision=prec, cfl=0.5)
    b.load(tmp_path / "c.ckpt")
    assert b.sync().steps == 7
    b.step(9)
    assert b.sync().t == a.sync().t
    assert np.array_equal(a.get_state(layout="cons", interior=True), b.get_state(layout="cons", interior=True))


def test_fvb_keep_lmv(tmp_path):
    r = subprocess.run([str(BIN / "fvb_keep"), "40", "lmv", "0.1", "--t-end", "0.05"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "FINAL L2 ERRORS" in r.stdout
    for k in range(11):
        w, h = _png(tmp_path / "figures" / ("keep_lmv_%04d.png" % k))
        assert (w, h) == (80, 40)


def _frame_fields_host(Q, g, h):
    """fv_up7's frame fields from an FP32 padded primitive state, restated in
    numpy (fv_up7_ducros_2d.cu:511-526, :800-829)."""
    n = Q.shape[-1] - 2 * g
    c = lambda q, dj, di: Q[q, g + dj:g + dj + n, g + di:g + di + n]
    duc = lambda pa, pb: (pb - pa) ** 2 / ((pb - pa) ** 2 + np.float32(0.1) * (pb + pa) ** 2)
    p = c(3, 0, 0)
    sd = np.maximum(np.maximum(duc(p, c(3, 0, 1)), duc(c(3, 0, -1), p)),
                    np.maximum(duc(p, c(3, 1, 0)), duc(c(3, -1, 0), p)))
    if g >= 3:
        w6 = [(-3, -1.0), (-2, 9.0), (-1, -45.0), (1, 45.0), (2, -9.0), (3, 1.0)]
        dvdx = sum(np.float32(k) * c(2, 0, o) for o, k in w6)
        dudy = sum(np.float32(k) * c(1, o, 0) for o, k in w6)
        vort = (dvdx - dudy) / np.float32(60.0 * h)
    else:  # two ghost layers: 4th-order central differences
        w4 = [(-2, 1.0), (-1, -8.0), (1, 8.0), (2, -1.0)]
        dvdx = sum(np.float32(k) * c(2, 0, o) for o, k in w4)
        dudy = sum(np.float32(k) * c(1, o, 0) for o, k in w4)
        vort = (dvdx - dudy) / np.float32(12.0 * h)
    speed = np.sqrt(c(1, 0, 0) ** 2 + c(2, 0, 0) ** 2)
    return {"rho": c(0, 0, 0), "vorticity": vort, "ducros": sd, "speed": speed, "p": p}


def test_frame_fields_of_the_two_ghost_layer_families():
    """KEEP and rec3 keep two ghost layers: the frame's vorticity is the
    4th-order central difference there"""
    for flux, case, n in (("keep", "lmv", 64), ("rec3", "gresho", 64)):
        s = F.Solver(n, flux=flux, bc="periodic", cfl=0.4)
        s.init_case(case)
        s.step(5)
        Q = s.get_state(dtype=np.float32)
        s.frame_begin()
        fr = s.frame_end()
        assert s.g == 2
        ref = _frame_fields_host(Q, 2, 1.0 / n)
        scale = float(np.abs(ref["vorticity"]).max())
        assert scale > 1.0  # a vortex: the panel is not empty
        assert np.abs(fr["vorticity"] - ref["vorticity"]).max() <= 1e-5 * scale, flux
        assert np.allclose(fr["rho"], ref["rho"], rtol=2e-6, atol=1e-7)


@pytest.mark.parametrize("case,bc,prec", [("sod", "reflect", "f64"), ("kh", "periodic", "f32c"),
                                          ("vortex", "periodic", "f32")])
def test_device_frame_fields_match_host_restatement(case, bc, prec):
    n = 96
    kw = dict(x0=-5, y0=-5, length=10.0) if case == "vortex" else {}
    s = F.Solver(n, bc=bc, precision=prec, cfl=0.4, **kw)
    s.init_case(case)
    s.step(20)
    Q = s.get_state(dtype=np.float32)   # the state the frame sees
    s.frame_begin()
    s.step(7)                           # overlaps the frame's copy
    fr = s.frame_end()
    ref = _frame_fields_host(Q, s.g, 10.0 / n if case == "vortex" else 1.0 / n)
    for k in ("rho", "p", "speed", "ducros"):
        assert np.allclose(fr[k], ref[k], rtol=2e-6, atol=1e-7), k
    scale = max(float(np.abs(ref["vorticity"]).max()), 1e-6)
    assert np.abs(fr["vorticity"] - ref["vorticity"]).max() <= 1e-5 * scale
    assert s.sync().steps == 27


def test_fvb_rec3_matches_the_oracle(tmp_path):
    """fvb_rec3 (fv_rec3's command line): step count, the limiter's mean-fix
    count and the L2 errors / minimum density it prints, against the oracle
    run to the same time"""
    import re
    import oracle as O
    for case, args, t_end in (("pv", ["32", "pv"], 0.3), ("sod", ["32"], 0.05)):
        r = subprocess.run([str(BIN / "fvb_rec3"), *args, "--t-end", str(t_end)], cwd=tmp_path,
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        out = r.stdout
        steps = int(re.search(r"Done: (\d+) steps", out).group(1))
        fixes = int(re.search(r"brutal mean-fix activations: (\d+)", out).group(1))
        assert "conservation drift: mass" in out
        L = 10.0 if case == "pv" else 1.0
        n, h = 32, L / 32
        U = O.rec3_ic(n, h, case)
        brutal0 = O.rec3_limit(U, n)
        O.bc(U, n, 2, 1)
        st, t, k, lmax, dt, brutal = O.rec3_run(U, n, h, 0.4, 10 ** 6, t_stop=t_end)
        assert st == 0 and k == steps and fixes == brutal0 + brutal
        if case == "pv":
            e_rho, e_vel = O.rec3_err(U, n, h, "pv")
            got_rho = float(re.search(r"L2\(rho\) = (\S+)", out).group(1))
            got_vel = float(re.search(r"L2\(vel\) = (\S+)", out).group(1))
            assert got_rho == pytest.approx(e_rho, rel=1e-5) and got_vel == pytest.approx(e_vel, rel=1e-5)
        else:
            rmin = float(U[0, 2:-2, 2:-2].min())
            got = float(re.search(r"final min rho = (\S+)", out).group(1))
            assert got == pytest.approx(rmin, rel=1e-3)
