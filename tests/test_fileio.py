"""Wavelet coefficient files (the reference's s2dw_fileio_mod, FITS and Matlab
formats): round trips through the C ABI, the byte layout checked by an
independent parser written here in numpy (FITS standard 4.0: 2880-byte
blocks, 80-character cards, big-endian IEEE doubles), the Matlab layout the
reference's reader relies on (src/mod/s2dw_fileio_mod.f90:637-763: 19 header
lines, five parameters, two skipped lines, three size lines per scale), and
the reference's error cases.  No GPU."""
import os

import numpy as np
import pytest

from s2dw_b200 import fileio
from s2dw_b200._lib import S2DWError
from s2dw_b200.core import band_limits, s2dw_core_comp_Jmax, wav_scale_shape

B, N, ALPHA = 16, 3, 2.0
J = s2dw_core_comp_Jmax(B, ALPHA)
BS = 3


def _coeffs(seed=0, J=J, B=B, N=N, alpha=ALPHA, bs=BS):
    rng = np.random.default_rng(seed)
    wavdyn = [np.asfortranarray(rng.standard_normal(wav_scale_shape(j, B, N, alpha)) * 10.0 ** rng.integers(-5, 5))
              for j in range(J + 1)]
    sc = np.asfortranarray(rng.standard_normal((bs, bs)) + 1j * rng.standard_normal((bs, bs)))
    return wavdyn, sc


def _static(wavdyn, J=J, B=B, N=N):
    w = np.zeros((J + 1, 2 * B - 1, 2 * B, N), order="F")
    for j, c in enumerate(wavdyn):
        w[j, :c.shape[0], :c.shape[1], :] = c
    return w


# ---------------------------------------------------------------------------
# an independent FITS reader (test infrastructure)
# ---------------------------------------------------------------------------
def _parse_fits(path):
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    pos, hdus = 0, []
    while pos < len(raw):
        cards = []
        while True:
            blk = raw[pos:pos + 2880]
            pos += 2880
            assert all(32 <= b < 127 for b in blk), "header must be printable ASCII"
            done = False
            for i in range(36):
                c = blk[80 * i:80 * i + 80].decode()
                cards.append(c)
                if c[:8].strip() == "END":
                    done = True
                    break
            if done:
                break
        kv = {}
        for c in cards:
            if c[8:10] == "= ":
                v = c[10:]
                if v.lstrip().startswith("'"):
                    v = v.lstrip()[1:]
                    v = v[:v.index("'")].rstrip()
                else:
                    v = v.split("/")[0].strip()
                kv.setdefault(c[:8].strip(), v)
        naxes = [int(kv[f"NAXIS{i}"]) for i in range(1, int(kv["NAXIS"]) + 1)]
        n = int(np.prod(naxes)) if naxes else 0
        nbytes = abs(int(kv["BITPIX"])) // 8 * n
        data = np.frombuffer(raw[pos:pos + nbytes], dtype=">f8") if kv["BITPIX"] == "-64" else raw[pos:pos + nbytes]
        pos += -(-nbytes // 2880) * 2880
        hdus.append((cards, kv, naxes, data))
    return hdus


def test_fits_round_trip_dynamic_and_static(tmp_path):
    wavdyn, sc = _coeffs(1)
    f1 = str(tmp_path / "wav_dyn.fits")
    fileio.s2dw_fileio_fits_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, f1, comment="round trip")
    w, s, J2, B2, N2, bs2, a2 = fileio.s2dw_fileio_fits_wav_read(f1)
    assert (J2, B2, N2, bs2, a2) == (J, B, N, BS, ALPHA)
    for j in range(J + 1):
        np.testing.assert_array_equal(w[j], wavdyn[j])
    np.testing.assert_array_equal(s, sc)
    ws, s_, *_ = fileio.s2dw_fileio_fits_wav_read(f1, dynamic=False)
    np.testing.assert_array_equal(ws, _static(wavdyn))
    np.testing.assert_array_equal(s_, sc)
    # the static writer writes the same file content (the DATE card aside)
    f2 = str(tmp_path / "wav_static.fits")
    fileio.s2dw_fileio_fits_wav_write(_static(wavdyn), sc, J, B, N, BS, ALPHA, f2, comment="round trip")
    h1, h2 = _parse_fits(f1), _parse_fits(f2)
    assert len(h1) == len(h2)
    for a, b in zip(h1, h2):
        assert a[2] == b[2]
        np.testing.assert_array_equal(a[3], b[3])


def test_fits_layout_independent_parser(tmp_path):
    wavdyn, sc = _coeffs(2)
    f = str(tmp_path / "w.fits")
    fileio.s2dw_fileio_fits_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, f)
    hdus = _parse_fits(f)
    # primary + SCOEFF_REAL + SCOEFF_IMAG + one WAV per scale (fileio:1333-1340)
    assert len(hdus) == 1 + 2 + (J + 1)
    cards, kv, naxes, _ = hdus[0]
    assert cards[0][:30] == "SIMPLE  =                    T"
    assert (kv["BITPIX"], kv["NAXIS"], kv["EXTEND"]) == ("-64", "0", "T")
    assert (int(kv["J"]), int(kv["B"]), int(kv["N"]), int(kv["BLSCOEFF"])) == (J, B, N, BS)
    assert float(kv["ALPHA"]) == ALPHA
    jcard = next(c for c in cards if c.startswith("J       ="))
    assert jcard[10:30] == f"{J:20d}"  # fixed format: right-justified to column 30
    for part, name in ((0, "SCOEFF_REAL"), (1, "SCOEFF_IMAG")):
        c, k, nx, d = hdus[1 + part]
        assert c[0].startswith("XTENSION= 'IMAGE   '")
        assert k["EXTNAME"] == name and nx == [BS, BS]
        want = sc.real if part == 0 else sc.imag
        np.testing.assert_array_equal(d.reshape(BS, BS, order="F"), want)
    for j in range(J + 1):
        c, k, nx, d = hdus[3 + j]
        bl, _ = band_limits(j, B, ALPHA)
        assert k["EXTNAME"] == "WAV" and nx == [2 * bl - 1, 2 * bl, N]
        np.testing.assert_array_equal(d.reshape(nx, order="F"), wavdyn[j])


def _write_foreign_fits(path, hdus):
    """A FITS file from (cards, raw data bytes) pairs, as another writer
    (CFITSIO) might lay it out: header padded with spaces, data with zeros."""
    out = b""
    for cards, data in hdus:
        h = "".join(c.ljust(80)[:80] for c in cards + ["END"])
        h += " " * (-len(h) % 2880)
        out += h.encode() + data + b"\0" * (-len(data) % 2880)
    open(path, "wb").write(out)


def test_fits_reads_other_bitpix_and_scaling(tmp_path):
    """ftg3dd converts any BITPIX with BSCALE/BZERO to double: so does the reader."""
    Jl, Bl, Nl, al = 1, 2, 1, 2.0  # bl = 2, 2 at both scales: cubes 3 x 4 x 1
    rng = np.random.default_rng(3)
    ints = [rng.integers(-1000, 1000, size=(3, 4, 1)).astype(">i4") for _ in range(Jl + 1)]
    prim = ["SIMPLE  =                    T", "BITPIX  =                  -64", "NAXIS   =                    0",
            "EXTEND  =                    T", "J       =                    1", "B       =                    2",
            "N       =                    1", "BLSCOEFF=                    1",
            "ALPHA   =      2.00000000D+00 / Fortran D exponent"]
    sc_r = np.array([1.5], dtype=">f4")
    sc_i = np.array([-0.25], dtype=">f4")

    def img(bitpix, shape, extra):
        return (["XTENSION= 'IMAGE   '", f"BITPIX  = {bitpix:20d}", f"NAXIS   = {len(shape):20d}"]
                + [f"NAXIS{i + 1:<3d}= {s:20d}" for i, s in enumerate(shape)]
                + ["PCOUNT  =                    0", "GCOUNT  =                    1"] + extra)

    hdus = [(prim, b""), (img(-32, [1, 1], ["EXTNAME = 'SCOEFF_REAL'"]), sc_r.tobytes()),
            (img(-32, [1, 1], ["EXTNAME = 'SCOEFF_IMAG'"]), sc_i.tobytes())]
    for j in range(Jl + 1):
        hdus.append((img(32, [3, 4, 1], ["BSCALE  =                 0.5", "BZERO   =                 10.",
                                         "EXTNAME = 'WAV     '"]), ints[j].tobytes(order="F")))
    f = str(tmp_path / "foreign.fits")
    _write_foreign_fits(f, hdus)
    w, s, J2, B2, N2, bs2, a2 = fileio.s2dw_fileio_fits_wav_read(f)
    assert (J2, B2, N2, bs2, a2) == (Jl, Bl, Nl, 1, al)
    assert s[0, 0] == 1.5 - 0.25j
    for j in range(Jl + 1):
        np.testing.assert_array_equal(w[j], 10.0 + 0.5 * ints[j].astype(np.float64))


def test_fits_error_cases(tmp_path):
    wavdyn, sc = _coeffs(4)
    f = str(tmp_path / "e.fits")
    fileio.s2dw_fileio_fits_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, f)
    with pytest.raises(S2DWError) as e:  # the writer refuses an existing file (fileio:986-992)
        fileio.s2dw_fileio_fits_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, f)
    assert e.value.code == 14
    with pytest.raises(S2DWError) as e:  # missing file (fileio:1311-1316)
        fileio.s2dw_fileio_fits_wav_read(str(tmp_path / "missing.fits"))
    assert e.value.code == 14
    # one HDU short: wrong number of headers (fileio:1333-1340)
    hdus = _parse_fits(f)
    raw = open(f, "rb").read()
    last = hdus[-1]
    nb = len(last[0]) * 80
    cut = len(raw) - (-(-nb // 2880) * 2880) - (-(-last[3].nbytes // 2880) * 2880)
    short = str(tmp_path / "short.fits")
    open(short, "wb").write(raw[:cut])
    with pytest.raises(S2DWError) as e:
        fileio.s2dw_fileio_fits_wav_read(short)
    assert e.value.code == 14
    # a NaN wavelet coefficient is a null value (fileio:1420-1424)
    bad = [w.copy(order="F") for w in wavdyn]
    bad[1][0, 0, 0] = np.nan
    fn = str(tmp_path / "nan.fits")
    fileio.s2dw_fileio_fits_wav_write(bad, sc, J, B, N, BS, ALPHA, fn)
    with pytest.raises(S2DWError) as e:
        fileio.s2dw_fileio_fits_wav_read(fn)
    assert e.value.code == 14


# ---------------------------------------------------------------------------
# Matlab format
# ---------------------------------------------------------------------------
def _e27_20(v):
    """Fortran E27.20 output of v (independent restatement for the test)."""
    if v == 0.0:
        return "0.00000000000000000000E+00".rjust(27)
    s = f"{abs(v):.19e}"
    mant, ex = s.split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    tail = f"E{'-' if e < 0 else '+'}{abs(e):02d}" if abs(e) <= 99 else f"{'-' if e < 0 else '+'}{abs(e):03d}"
    return (("-" if v < 0 else "") + "0." + digits + tail).rjust(27)


def test_matlab_round_trip_and_layout(tmp_path):
    wavdyn, sc = _coeffs(5)
    wavdyn[0][0, 0, 0] = 1e-120   # three-digit exponents
    wavdyn[0][1, 0, 0] = -3.25e150
    wavdyn[0][2, 0, 0] = 0.0
    m = str(tmp_path / "wcoeff_test.m")
    fileio.s2dw_fileio_matlab_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, m, comment="layout")
    w, s, J2, B2, N2, bs2, a2 = fileio.s2dw_fileio_matlab_wav_read(m)
    assert (J2, B2, N2, bs2, a2) == (J, B, N, BS, ALPHA)
    for j in range(J + 1):
        np.testing.assert_array_equal(w[j], wavdyn[j])
    tri = np.tril(np.ones((BS, BS), dtype=bool))
    np.testing.assert_array_equal(s[tri], sc[tri])   # the format stores the lower triangle
    assert not s[~tri].any()
    ws, *_ = fileio.s2dw_fileio_matlab_wav_read(m, dynamic=False)
    np.testing.assert_array_equal(ws, _static(wavdyn))

    lines = open(m).read().split("\n")
    assert lines[0].startswith("function [J, N, B, bl_scoeff, alpha, scoeff, wcoeff] = wcoeff_test")
    # the reference's reader: skip 19 lines, five parameters, skip 2, sizes
    assert lines[19] == "J         = " + f"{J:27d}" + ";"
    assert lines[20] == "N         = " + f"{N:27d}" + ";"
    assert lines[21] == "B         = " + f"{B:27d}" + ";"
    assert lines[22] == "bl_scoeff = " + f"{BS:27d}" + ";"
    assert lines[23] == "alpha     = " + _e27_20(ALPHA) + ";"
    for j in range(J + 1):
        bl, _ = band_limits(j, B, ALPHA)
        assert lines[26 + 3 * j] == f"wcoeff_size_aa({j + 1:5d}) = {2 * bl - 1:15d};"
        assert lines[27 + 3 * j] == f"wcoeff_size_bb({j + 1:5d}) = {2 * bl:15d};"
        assert lines[28 + 3 * j] == f"wcoeff_size_gg({j + 1:5d}) = {N:15d};"
    base = m[:-2]
    sl = open(base + "_scoeff.dat").read().split("\n")[:-1]
    want = [_e27_20(sc[el, mm].real) for el in range(BS) for mm in range(el + 1)]
    want += [_e27_20(sc[el, mm].imag) for el in range(BS) for mm in range(el + 1)]
    assert sl == want
    wl = open(base + "_wcoeff.dat").read().split("\n")[:-1]
    assert wl == [_e27_20(x) for c in wavdyn for x in c.ravel(order="F")]
    # 20 significant digits of the doubles nearest 1e-120 and -3.25e150
    assert wl[0] == " 0.99999999999999997861-120"
    assert wl[1] == "-0.32500000000000001649+151"


def test_matlab_reads_fortran_written_values(tmp_path):
    """Values as gfortran writes them (E, D and letterless exponents) in a
    file laid out as the reference's writer lays it out."""
    Jl, Bl, Nl, al, bs = 1, 2, 1, 2.0, 1
    rng = np.random.default_rng(6)
    cubes = [rng.standard_normal((3, 4, 1)) for _ in range(Jl + 1)]
    base = str(tmp_path / "ref")
    head = ["function [J, N, B, bl_scoeff, alpha, scoeff, wcoeff] = ref"] + ["%"] * 16 + [""]
    body = ["% Size parameters", "J         = " + f"{Jl:27d};", "N         = " + f"{Nl:27d};",
            "B         = " + f"{Bl:27d};", "bl_scoeff = " + f"{bs:27d};", "alpha     =  0.20000000000000000000D+01;",
            "", "% Wavelet coefficient array sizes"]
    for j in range(Jl + 1):
        body += [f"wcoeff_size_aa({j + 1:5d}) = {3:15d};", f"wcoeff_size_bb({j + 1:5d}) = {4:15d};",
                 f"wcoeff_size_gg({j + 1:5d}) = {1:15d};"]
    open(base + ".m", "w").write("\n".join(head + body) + "\n")
    open(base + "_scoeff.dat", "w").write(_e27_20(0.5) + "\n" + _e27_20(-2.0) + "\n")
    vals = [x for c in cubes for x in c.ravel(order="F")]
    open(base + "_wcoeff.dat", "w").write("\n".join(_e27_20(x) for x in vals) + "\n")
    w, s, J2, B2, N2, bs2, a2 = fileio.s2dw_fileio_matlab_wav_read(base + ".m")
    assert (J2, B2, N2, bs2, a2) == (Jl, Bl, Nl, bs, al)
    assert s[0, 0] == 0.5 - 2.0j
    for j in range(Jl + 1):
        np.testing.assert_array_equal(w[j], cubes[j])


def test_matlab_error_cases(tmp_path):
    wavdyn, sc = _coeffs(7)
    m = str(tmp_path / "x.m")
    fileio.s2dw_fileio_matlab_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, m)
    with pytest.raises(S2DWError) as e:  # status='new' in the reference's open
        fileio.s2dw_fileio_matlab_wav_write(wavdyn, sc, J, B, N, BS, ALPHA, m)
    assert e.value.code == 14
    with pytest.raises(S2DWError) as e:
        fileio.s2dw_fileio_matlab_wav_read(str(tmp_path / "none.m"))
    assert e.value.code == 14
    os.remove(m[:-2] + "_wcoeff.dat")
    with pytest.raises(S2DWError) as e:
        fileio.s2dw_fileio_matlab_wav_read(m)
    assert e.value.code == 14
