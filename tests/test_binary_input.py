"""The binary input form (ufem_convert_input, read by ufem_read_input and the
Monte Carlo plugin): CPU checks of the file against the model tables with an
independent numpy reader, and (GPU) identical models and outputs from the
text and the binary form of the same input."""
import os

import numpy as np
import pytest

from golden_util import load, model_from

CASES = ["mc_out_plate_6x3", "mc_out_beam_4x2x2", "mc_beam_4x2x2"]
ORDER = ["rsID", "rsType", "rsFrom", "rsVal", "mpID", "mpType", "mpFrom", "mpVal", "nID", "nx", "ny", "nz",
         "eID", "eType", "eRS", "eMP", "eFrom", "eNodes", "nlNode", "nlType", "nlDir", "nlVal", "mc_len",
         "mc_pos", "mc_type", "mc_item", "mc_sub", "mc_iter"]
FLOATS = {"rsVal", "mpVal", "nx", "ny", "nz", "nlVal"}


def _read_binary(path):
    b = open(path, "rb").read()
    assert b[:8] == b"UFEMBIN1"
    assert np.frombuffer(b, "<u4", 1, 8)[0] == 0x01020304
    off, out = 12, {}
    for name in ORDER:
        n = int(np.frombuffer(b, "<i8", 1, off)[0])
        off += 8
        out[name] = np.frombuffer(b, "<f8" if name in FLOATS else "<i8", n, off).copy()
        off += 8 * n
    assert off == len(b)
    return out


def _files(tmp_path, name):
    from ufem_b200 import meshgen as mg
    z = load(name)
    m = model_from(z)
    txt, binp = str(tmp_path / f"{name}.fem"), str(tmp_path / f"{name}.bin")
    mg.write_fem(m, txt)
    return z, m, txt, binp


@pytest.mark.parametrize("name", CASES)
def test_binary_holds_the_tables(tmp_path, name):
    from ufem_b200.api import convert_input
    z, m, txt, binp = _files(tmp_path, name)
    convert_input(txt, binp)
    t = _read_binary(binp)
    np.testing.assert_array_equal(np.stack([t["nx"], t["ny"], t["nz"]], 1), m.n_xyz)
    np.testing.assert_array_equal(t["eType"], m.e_type)
    np.testing.assert_array_equal(t["eRS"], m.e_rs)
    np.testing.assert_array_equal(t["eMP"], m.e_mp)
    np.testing.assert_array_equal(t["eNodes"], m.e_nodes.ravel())
    np.testing.assert_array_equal(t["eFrom"], m.e_from())
    np.testing.assert_array_equal(t["mpType"], m.mp_type)
    np.testing.assert_array_equal(t["mpVal"], np.concatenate(m.mp_vals))
    np.testing.assert_array_equal(t["rsType"], m.rs_type)
    np.testing.assert_array_equal(t["nlNode"], m.nl_node)
    np.testing.assert_array_equal(t["nlType"], m.nl_type)
    np.testing.assert_array_equal(t["nlDir"], m.nl_dir)
    np.testing.assert_array_equal(t["nlVal"], m.nl_val)
    np.testing.assert_array_equal(t["mc_len"], [m.mc_ilen, m.mc_olen])
    mv = np.stack([t["mc_pos"], t["mc_type"], t["mc_item"], t["mc_sub"], t["mc_iter"]], 1)
    np.testing.assert_array_equal(mv, m.mc_vars)
    # binary -> binary is the identity
    again = str(tmp_path / "again.bin")
    convert_input(binp, again)
    assert open(again, "rb").read() == open(binp, "rb").read()


def test_damaged_binary_is_rejected(tmp_path):
    from ufem_b200 import _lib
    from ufem_b200.api import convert_input
    _, _, txt, binp = _files(tmp_path, CASES[0])
    convert_input(txt, binp)
    b = open(binp, "rb").read()
    cut = str(tmp_path / "cut.bin")
    open(cut, "wb").write(b[: len(b) // 2])
    with pytest.raises(_lib.UfemError):
        convert_input(cut, str(tmp_path / "x.bin"))
    bad = bytearray(b)
    bad[8:12] = (0x04030201).to_bytes(4, "little")  # another byte order
    open(cut, "wb").write(bytes(bad))
    with pytest.raises(_lib.UfemError):
        convert_input(cut, str(tmp_path / "x.bin"))


def _write_binary(path, t):
    parts = [b"UFEMBIN1", np.array([0x01020304], "<u4").tobytes()]
    for name in ORDER:
        a = np.asarray(t[name], "<f8" if name in FLOATS else "<i8")
        parts += [np.array([a.size], "<i8").tobytes(), a.tobytes()]
    open(path, "wb").write(b"".join(parts))


def _rejected(src, tmp_path):
    from ufem_b200 import _lib
    from ufem_b200.api import convert_input
    with pytest.raises(_lib.UfemError):
        convert_input(src, str(tmp_path / "x.bin"))


def test_malformed_element_and_value_ranges_are_rejected(tmp_path):
    """Both readers check every element's node count against its type and
    the order of the real-set and material value ranges before any table is
    indexed (host only: the checks run in ufem_convert_input too)."""
    from ufem_b200.api import convert_input
    _, _, txt, binp = _files(tmp_path, "mc_out_beam_4x2x2")
    convert_input(txt, binp)
    t = _read_binary(binp)
    bad = str(tmp_path / "bad.bin")
    # the last brick loses a node: the list ends one entry early
    tt = dict(t, eNodes=t["eNodes"][:-1])
    _write_binary(bad, tt)
    _rejected(bad, tmp_path)
    # an element start out of order
    ef = t["eFrom"].copy()
    ef[2], ef[3] = ef[3], ef[2]
    _write_binary(bad, dict(t, eFrom=ef))
    _rejected(bad, tmp_path)
    # material value ranges out of order
    mf = t["mpFrom"].copy()
    if mf.size >= 2:
        mf[0], mf[1] = mf[1], mf[0]
        _write_binary(bad, dict(t, mpFrom=mf))
        _rejected(bad, tmp_path)
    # the unchanged tables still pass
    _write_binary(bad, t)
    convert_input(bad, str(tmp_path / "ok.bin"))
    # text form: the first of two bricks declares 7 nodes (the list length 15
    # matches the counts, so only the per-element check can catch it)
    from ufem_b200 import meshgen as mg
    good = str(tmp_path / "two.fem")
    mg.write_fem(mg.beam_brick(2, 1, 1, 2.0, 1.0, 1.0), good)
    convert_input(good, str(tmp_path / "two.bin"))
    body = open(good).read()
    assert "1 9 0 0 8\n2 9 0 0 8\n16\n0 1 4 3 6 7 10 9\n" in body
    body = body.replace("1 9 0 0 8\n2 9 0 0 8\n16\n0 1 4 3 6 7 10 9\n",
                        "1 9 0 0 7\n2 9 0 0 8\n15\n0 1 4 3 6 7 10\n")
    badtxt = str(tmp_path / "bad.fem")
    open(badtxt, "w").write(body)
    _rejected(badtxt, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_binary_and_text_give_the_same_model(tmp_path, name):
    """Same DOF numbering and bitwise the same static solution from either form."""
    from ufem_b200.api import GpuModel, convert_input
    z, m, txt, binp = _files(tmp_path, name)
    convert_input(txt, binp)
    gt, gb = GpuModel(path=txt), GpuModel(path=binp)
    np.testing.assert_array_equal(gt.ndoffld(m.nLen), gb.ndoffld(m.nLen))
    rt, _ = gt.fem_solve()
    rb, _ = gb.fem_solve()
    assert rt == 0 and rb == 0
    assert np.array_equal(gt.u(), gb.u())


@pytest.mark.gpu
def test_plugin_reads_the_binary_form(tmp_path):
    """monte_init_lib_stuff on the binary file: the same outputs, bit for bit."""
    from ufem_b200.api import convert_input
    from ufem_b200.mc import MonteLib
    z, m, txt, binp = _files(tmp_path, "mc_out_beam_4x2x2")
    convert_input(txt, binp)
    outs = []
    for path in (txt, binp):
        lib = MonteLib(path)
        try:
            rv, o, st = lib.solution_batch(z["ifld"])
            assert rv == 0 and (st == 0).all()
            outs.append(o)
        finally:
            lib.close()
    assert np.array_equal(outs[0], outs[1])
