"""CPU: the ILDG/LIME reader and the known answers defined on the reference's
ILDG test configuration ildg_io/conf.00200.

* the reader against files written here by an independent writer (64- and
  32-bit data, direction mapping, SciDAC checksum: recorded, corrupted, absent);
* conf.00200 as decoded by the reader (tests/golden/conf00200.npz): its recorded
  plaquette and checksum, and -- where the reference tree is present -- a fresh
  decode equal to the fixture;
* the second blocks of physics/fermionmatrix/explicit_test.cpp (M_wilson,
  M_tm_plus, M_tm_minus on conf.00200) and fermionmatrix_test.cpp (the five eo
  matrices on conf.00200) through both oracle builds, at the reference's 0.01 %.
"""
import json
import os
import struct
import zlib

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLD, "reference_kats.json")))
CONF = np.load(os.path.join(GOLD, "conf00200.npz"))
BACKENDS = ["port", "reference"]
FM = {"Aee": "OP_AEE", "Aee_minus": "OP_AEE_MINUS", "Qplus_eo": "OP_QPLUS_EO", "Qminus_eo": "OP_QMINUS_EO",
      "QplusQminus_eo": "OP_QPQM_EO"}


def _oracle(request, kind):
    return request.getfixturevalue("port" if kind == "port" else "ref")


def _lime_record(typ: str, payload: bytes, mb: bool, me: bool) -> bytes:
    flags = (0x8000 if mb else 0) | (0x4000 if me else 0)
    head = struct.pack(">IHHQ", 0x456789AB, 1, flags, len(payload)) + typ.encode().ljust(128, b"\0")
    return head + payload + b"\0" * ((8 - len(payload) % 8) % 8)


def _write_ildg(path, ildg_links, ns, nt, prec=64, checksum="good"):
    """ildg_links: (V, 4, 3, 3) complex in ILDG order (site x fastest, direction x, y, z, t)."""
    V = ns ** 3 * nt
    dt = ">f8" if prec == 64 else ">f4"
    raw = np.empty((V, 4, 3, 3, 2))
    raw[..., 0], raw[..., 1] = ildg_links.real, ildg_links.imag
    data = raw.astype(dt).tobytes()
    fmt = (f"<?xml version=\"1.0\"?><ildgFormat><version>1.0</version><field>su3gauge</field>"
           f"<precision>{prec}</precision><lx>{ns}</lx><ly>{ns}</ly><lz>{ns}</lz><lt>{nt}</lt></ildgFormat>")
    site = len(data) // V
    a = b = 0
    for r in range(V):
        c = zlib.crc32(data[r * site:(r + 1) * site]) & 0xFFFFFFFF
        ra, rb = r % 29, r % 31
        a ^= ((c << ra) | (c >> (32 - ra))) & 0xFFFFFFFF if ra else c
        b ^= ((c << rb) | (c >> (32 - rb))) & 0xFFFFFFFF if rb else c
    if checksum == "bad":
        a ^= 1
    recs = [_lime_record("xlf-info", b"plaquette = 0.5\n", True, False),
            _lime_record("ildg-format", fmt.encode(), False, False),
            _lime_record("ildg-binary-data", data, False, checksum == "none")]
    if checksum != "none":
        sc = f"<scidacChecksum><version>1.0</version><suma>{a:x}</suma><sumb>{b:x}</sumb></scidacChecksum>"
        recs.append(_lime_record("scidac-checksum", sc.encode(), False, True))
    with open(path, "wb") as f:
        f.write(b"".join(recs))
    return a, b


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("checksum", ["good", "bad", "none"])
def test_reader_round_trip(tmp_path, prec, checksum):
    import cl2qcd_b200 as c2q
    ns, nt = 4, 8
    V = ns ** 3 * nt
    rng = np.random.default_rng(prec + len(checksum))
    links = rng.standard_normal((V, 4, 3, 3)) + 1j * rng.standard_normal((V, 4, 3, 3))
    path = str(tmp_path / "cfg.lime")
    a, b = _write_ildg(path, links, ns, nt, prec, checksum)
    rns, rnt, aos, info = c2q.host.read_ildg(path)
    assert (rns, rnt, info["precision"]) == (ns, nt, prec)
    assert info["checksum_status"] == {"good": 1, "bad": 0, "none": -1}[checksum]
    if checksum == "good":
        assert (info["suma"], info["sumb"]) == (a, b)
    # ILDG direction l is stored as mu = (l + 1) % 4 at link mu + 4 * site
    expect = np.empty((4 * V, 18))
    m = links.astype(np.complex64) if prec == 32 else links
    for l in range(4):
        mu = (l + 1) % 4
        blk = np.stack([m[:, l].real, m[:, l].imag], axis=-1).reshape(V, 18)
        expect[mu::4] = blk
    assert np.array_equal(aos, expect)
    assert "plaquette = 0.5" in info["xlf_info"]


@pytest.mark.parametrize("damage", ["truncated", "huge_length", "wrapping_length"])
def test_reader_rejects_damaged_records(tmp_path, damage):
    """A record whose header claims more bytes than the file holds -- cut off,
    absurdly long, or long enough to wrap a 64-bit offset -- is refused."""
    import cl2qcd_b200 as c2q
    ns, nt = 4, 4
    V = ns ** 3 * nt
    links = np.ones((V, 4, 3, 3), dtype=complex)
    path = str(tmp_path / "cfg.lime")
    _write_ildg(path, links, ns, nt, 64, "good")
    raw = bytearray(open(path, "rb").read())
    if damage == "truncated":
        raw = raw[:len(raw) - 4000]
    else:  # the length field of the first record (bytes 8..16 of its header)
        n = (1 << 62) if damage == "huge_length" else (1 << 64) - 100
        raw[8:16] = struct.pack(">Q", n)
    bad = str(tmp_path / "bad.lime")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(Exception):
        c2q.host.read_ildg(bad)


def test_conf00200_fixture():
    import cl2qcd_b200 as c2q
    meta = KATS["ildg_conf00200"]
    assert (int(CONF["ns"]), int(CONF["nt"])) == (4, 4)
    assert meta["checksum_status"] == 1  # the file's SciDAC checksum matches its data
    g = CONF["gauge"]
    assert c2q.host.plaquette(c2q.Lattice(4, 4), g) == pytest.approx(meta["plaquette_recorded"], abs=5e-7)
    M = (g[:, 0::2] + 1j * g[:, 1::2]).reshape(-1, 3, 3)
    assert np.allclose(M @ np.conj(np.swapaxes(M, 1, 2)), np.eye(3), atol=1e-12)


def test_reader_on_reference_file():
    ref = os.environ.get("CL2QCD_REFERENCE", "")
    path = os.path.join(ref, "ildg_io", "conf.00200")
    if not ref or not os.path.exists(path):
        pytest.skip("reference tree not named by CL2QCD_REFERENCE, or absent")
    import cl2qcd_b200 as c2q
    ns, nt, aos, info = c2q.host.read_ildg(path)
    assert np.array_equal(aos, CONF["gauge"]) and info["checksum_status"] == 1


@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("name", sorted(KATS["explicit_conf00200"]))
def test_explicit_kats_on_conf00200(request, O, kind, name):
    o = _oracle(request, kind)
    kat = KATS["explicit_conf00200"][name]
    o.set_lattice(4, 4)
    g = CONF["gauge"]
    kappa, mubar = kat["kappa"], 2 * kat["kappa"] * kat["mu"]
    sf1 = o.pseudo_randomize(o.vol, kat["seeds"]["sf1"])
    op = {"M_wilson": lambda x: o.m_tm_plus(x, g, kappa, 0.0),
          "M_tm_plus": lambda x: o.m_tm_plus(x, g, kappa, mubar),
          "M_tm_minus": lambda x: o.m_tm_minus(x, g, kappa, mubar)}[kat["operator"]]
    sf2 = op(sf1)
    assert o.squarenorm_full(sf2) == pytest.approx(kat["refs"][0], rel=1e-4)
    sf1 = op(sf2)
    assert o.squarenorm_full(sf1) == pytest.approx(kat["refs"][1], rel=1e-4)


@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("name", sorted(FM))
def test_fermionmatrix_eo_kats_on_conf00200(request, O, kind, name):
    """fermionmatrix_test.cpp, second block: conf.00200, nTime 4, Wilson, kappa 0.125."""
    o = _oracle(request, kind)
    kat = KATS["fermionmatrix_eo"][name]
    o.set_lattice(4, 4)
    g = CONF["gauge"]
    src = o.pseudo_randomize(o.vol, kat["seed"])
    sf1, sf2 = o.convert_to_eo(src)
    op = getattr(O, FM[name])
    sf2 = o.apply(op, sf1, g, 0.125, 0.0, action=O.WILSON)
    assert o.squarenorm(sf2) == pytest.approx(kat["refs"][2], rel=1e-4)
    sf1 = o.apply(op, sf2, g, 0.125, 0.0, action=O.WILSON)
    assert o.squarenorm(sf1) == pytest.approx(kat["refs"][3], rel=1e-4)


@pytest.mark.parametrize("kind", BACKENDS)
def test_oracle_reproduces_inverter_reference_on_conf00200(request, O, kind):
    """executables/tests/inverter_test_ref2 (inverter_test_input_2: conf.00200, kappa 0.15,
    mu 4, twisted mass, 12 point sources, ps correlator along z, the default direction;
    compared at 0.1 %)."""
    o = _oracle(request, kind)
    ref = KATS["inverter"]["inverter_test_ref2"]
    ns, nt = 4, 4
    kappa, mu = float(ref["input"]["kappa"]), float(ref["input"]["mu"])
    o.set_lattice(ns, nt, 0.0, 0.0)
    g = CONF["gauge"]
    C = np.zeros(nt)
    for k in range(12):
        src = np.zeros((o.vol, 24))
        src[0, 2 * (3 * (k % 4) + k // 4)] = 1.0
        phi, _, _ = o.perform_inversion_eo(src, g, kappa, 2 * kappa * mu, O.TWISTEDMASS,
                                           O.SolverParams(prec=1e-23, cgmax=1000, solver=2))
        C += (phi ** 2).sum(axis=1).reshape(nt, ns, ns, ns).sum(axis=(0, 2, 3))  # along z, the default
    C *= (2 * kappa) ** 2 / (ns * ns * nt)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=ref["tolerance_percent"] / 100)
    np.testing.assert_allclose(C, ref["ps_correlator"], rtol=1e-9)
