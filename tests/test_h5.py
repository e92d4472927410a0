"""HDF5 files of the reference's layout (thor_b200/h5.py) against files the reference wrote.

tests/golden/h5/ holds three planet files written by the reference's storage layer (H5Cpp with
default properties; tests/golden/h5/make_fixtures.py copies them). The reader must return their
contents; the writer must produce files whose datasets carry the same object-header messages in
the same order, with the same datatype, dataspace and fill-value encodings, and that read back
to the same values.
"""
import io
import os

import numpy as np
import pytest

from thor_b200 import esp, h5

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "h5")


def golden(name):
    return os.path.join(GOLDEN, name)


# values pinned from the three files (the Earth Held-Suarez one is the glevel-4 / 32-level
# benchmark configuration: radius, gravity, gas constants, 36 km top, Diffc 0.0048)
PINNED = {
    "planet_earth_hs_g4L32.h5": dict(A=6371000.0, glevel=4, vlevel=32, Gravit=9.8, Rd=287.0,
                                     Cp=1005.0, Top_altitude=36000.0, Tmean=300.0, Diffc=0.0048,
                                     core_benchmark=1, P_Ref=100000.0, Omega=7.292e-05,
                                     spring_beta=1.15),
    "planet_deep_g4L40.h5": dict(A=94400000.0, glevel=4, vlevel=40, Gravit=9.42, Rd=4593.0,
                                 Cp=14308.4, Top_altitude=8000000.0, Tmean=1759.0,
                                 core_benchmark=4, P_Ref=22000000.0),
    "planet_earth_g5L20.h5": dict(A=6371000.0, glevel=5, vlevel=20, Top_altitude=10000.0,
                                  core_benchmark=7),
}


@pytest.mark.parametrize("name", sorted(PINNED))
def test_reader_on_reference_files(name):
    d = h5.read(golden(name))
    for k, v in PINNED[name].items():
        a, attrs = d[k]
        assert a.shape == (1,) and a[0] == v, (k, a, v)
        assert a.dtype == (np.int32 if isinstance(v, int) else np.float64), k
        assert set(attrs) == {"Variable", "units"}, k
    assert d["A"][1] == {"Variable": "Planet radius", "units": "m"}
    assert d["Rd"][1] == {"Variable": "Gas constant", "units": "J/(Kg K)"}


def rewrite(src, dst):
    w = h5.H5Writer(dst)
    for k, (a, at) in h5.read(src).items():
        w.table(k, a, at["units"], at["Variable"])
    w.close()


@pytest.mark.parametrize("name", sorted(PINNED))
def test_writer_matches_the_reference_layout(tmp_path, name):
    src, dst = golden(name), str(tmp_path / "out.h5")
    rewrite(src, dst)
    a, b = h5.read(src), h5.read(dst)
    assert set(a) == set(b)
    for k in a:
        assert a[k][0].dtype == b[k][0].dtype and np.array_equal(a[k][0], b[k][0]), k
        assert a[k][1] == b[k][1], k
    # same messages, in the same order, with the same datatype encodings; the reference's header
    # continuation messages (where a long description overflowed its first header block) aside
    sa, sb = h5.structure(src), h5.structure(dst)
    for k in sa:
        types_a = [t for t in sa[k][0] if t != h5.MSG_CONTINUATION]
        assert types_a == sb[k][0], (k, sa[k][0], sb[k][0])
        assert sa[k][1] == sb[k][1], k


def _group(d):
    """(B-tree address, heap address, heap header, {name: SNOD entry bytes}, SNOD headers) of the
    root group of file bytes d (superblock v0, root symbol-table entry cache)."""
    import struct
    bt, hp = struct.unpack_from("<QQ", d, 80)
    heap_data = struct.unpack_from("<Q", d, hp + 24)[0]
    used = struct.unpack_from("<H", d, bt + 6)[0]
    entries, snods = {}, []
    for i in range(used):
        child = struct.unpack_from("<Q", d, bt + 24 + 16 * i + 8)[0]
        snods.append(d[child:child + 6])
        for s in range(struct.unpack_from("<H", d, child + 6)[0]):
            e = d[child + 8 + 40 * s:child + 48 + 40 * s]
            name_off = struct.unpack_from("<Q", e)[0]
            name = d[heap_data + name_off:d.index(b"\0", heap_data + name_off)].decode()
            entries[name] = (name_off, e[16:40])
    return bt, hp, d[hp:hp + 8], entries, snods, d[bt:bt + 6]


@pytest.mark.parametrize("name", sorted(PINNED))
def test_writer_bytes_pinned_to_the_reference_files(tmp_path, name):
    """Byte-level pins against the files the library wrote: the superblock (signature, versions,
    sizes of offsets and lengths, group K values, base address, no free-space or driver block,
    the root symbol-table entry with its cached B-tree and heap addresses), the end-of-file address
    equal to the file length, the root object header, the group B-tree node header (type 0, leaf),
    the symbol-table node headers and entry format (cache type 0, empty scratch), and the local
    heap's packing of the names (the empty name, then each name null-terminated and 8-byte
    aligned, so the free block starts where the reference's does). Not pinned: the order of the
    names in the heap (the library's is creation order, the writer's sorted), how the library
    splits symbol-table nodes (4 to 8 entries each, where the writer fills them) and where it puts
    the heap's data and the objects after growing them."""
    import struct
    src, dst = golden(name), str(tmp_path / "out.h5")
    rewrite(src, dst)
    ref, out = open(src, "rb").read(), open(dst, "rb").read()
    assert out[:40] == ref[:40] and out[48:96] == ref[48:96]
    for d in (ref, out):
        assert struct.unpack_from("<Q", d, 40)[0] == len(d)
    root = struct.unpack_from("<Q", ref, 64)[0]
    assert out[root:root + 40] == ref[root:root + 40]
    gr, go = _group(ref), _group(out)
    assert (gr[0], gr[1]) == (go[0], go[1])                      # B-tree and heap addresses
    assert go[2] == gr[2] == b"HEAP\0\0\0\0"
    assert go[5][:4] == gr[5][:4] == b"TREE" and go[5][4:6] == gr[5][4:6] == b"\0\0"
    assert all(s[:6] == b"SNOD\x01\x00" for s in gr[4] + go[4])
    assert set(gr[3]) == set(go[3])
    packed = 8 + sum(-(-(len(n) + 1) // 8) * 8 for n in gr[3])    # the empty name, then each name
    for g in (gr, go):
        for n, (off, cache) in g[3].items():
            assert off % 8 == 0 and cache == b"\0" * 24, n       # aligned; cache type 0, no scratch
        slots = sorted(off for off, _ in g[3].values())
        assert slots[0] == 8 and len(set(slots)) == len(slots)
    free_ref = struct.unpack_from("<Q", ref, gr[1] + 16)[0]
    free_out = struct.unpack_from("<Q", out, go[1] + 16)[0]
    assert free_out == free_ref == packed


def test_writer_round_trip_many_and_large(tmp_path):
    """More datasets than one symbol-table node holds, long arrays, int32, awkward names and
    an empty unit string."""
    rng = np.random.default_rng(3)
    items = {}
    w = h5.H5Writer(str(tmp_path / "many.h5"))
    for i in range(61):
        name = ["a", "Z", "_x", "Mh", "mh", "A_b"][i % 6] + str(i)
        if i % 5 == 0:
            arr = rng.integers(-2**31, 2**31 - 1, size=i + 1).astype(np.int32)
        else:
            arr = rng.standard_normal(i * 37 + 1)
        unit = "" if i % 7 == 0 else "u%d" % i
        items[name] = (arr, unit, "description of %s" % name)
        w.table(name, arr, unit, "description of %s" % name)
    big = rng.standard_normal(1_500_000)
    w.table("/big", big, "kg", "a big table")
    w.value("/step", 12345, "-", "Step number")
    w.close()
    d = h5.read(str(tmp_path / "many.h5"))
    assert len(d) == 63
    for name, (arr, unit, desc) in items.items():
        assert np.array_equal(d[name][0], arr) and d[name][0].dtype == arr.dtype, name
        assert d[name][1] == {"Variable": desc, "units": unit}, name
    assert np.array_equal(d["big"][0], big)
    assert d["step"][0].dtype == np.int32 and d["step"][0][0] == 12345


class FakeContext:
    """What esp.write_state reads from a context: fields in the reference layout."""

    def __init__(self, N, nv):
        rng = np.random.default_rng(5)
        self.f = {n: rng.standard_normal(N * nv * k)
                  for n, k in (("Rho", 1), ("pressure", 1), ("Mh", 3), ("profx_Qheat", 1),
                               ("Rd", 1), ("Cp", 1))}
        self.f["Wh"] = rng.standard_normal(N * (nv + 1))

    def get(self, name):
        return self.f[name]


def test_state_file_names_units_and_restart_read(tmp_path):
    x = FakeContext(42, 5)
    c, _ = esp.read_config("", io.StringIO())
    path = str(tmp_path / "esp_output_Sim_3.h5")
    esp.write_state(path, x, 77, 4620.0, c, glob=(1.0, 2.0, 3.0, 4.0, 5.0, 6.0))
    d = h5.read(path)
    assert d["nstep"][0].dtype == np.int32 and d["nstep"][0][0] == 77
    assert d["Pressure"][1] == {"Variable": "Pressure", "units": "Pa"}
    assert d["Mh"][1] == {"Variable": "Horizontal Momentum", "units": "kg m^-2 s^-1"}
    assert d["GlobalMass"][0][0] == 2.0 and d["GlobalEnt"][0][0] == 6.0
    state, nstep, t = esp.read_state(path)
    assert nstep == 77 and t == 4620.0
    for f in ("Rho", "pressure", "Mh", "Wh", "Rd", "Cp"):
        assert np.array_equal(state[f], x.get(f)), f
    # restart naming (src/utils/directories.cpp:270-362)
    assert esp.output_numbering(path) == ("Sim", 3)
    assert esp.output_numbering(str(tmp_path / "esp_output_my_sim_12.h5")) == ("my_sim", 12)
    assert esp.output_numbering(str(tmp_path / "esp_initial.h5")) is None
    assert esp.planet_file(path, True) == str(tmp_path / "esp_output_planet_Sim.h5")
    assert esp.planet_file(str(tmp_path / "esp_initial.h5"), False) == \
        str(tmp_path / "esp_initial_planet.h5")
    assert esp.planet_file(str(tmp_path / "esp_initial.h5"), True) is None


def test_planet_file_check_against_reference_file():
    """The restart check reads the reference's own planet file: the Earth benchmark at glevel 4,
    32 levels passes, another level count fails."""
    c, _ = esp.read_config("radius = 6371000.0\nTop_altitude = 36000.0\nglevel = 4\n"
                           "vlevel = 32\n", io.StringIO())
    out = io.StringIO()
    assert esp.check_planet(golden("planet_earth_hs_g4L32.h5"), c, out), out.getvalue()
    c["vlevel"] = 48
    out = io.StringIO()
    assert not esp.check_planet(golden("planet_earth_hs_g4L32.h5"), c, out)
    assert "mismatch for /vlevel" in out.getvalue()


def test_planet_file_of_a_configuration(tmp_path):
    c, _ = esp.read_config("RayleighSponge = true\nradiative_transfer = true\n", io.StringIO())
    path = str(tmp_path / "p.h5")
    esp.write_planet(path, c)
    d = h5.read(path)
    assert d["nlat_bins"][0].dtype == np.int32 and d["nlat_bins"][0][0] == 20
    assert d["radiative_transfer"][0][0] == 1.0 and d["phy_module"][1]["Variable"] == "multi"
    # the names the reference's planet file has are all there
    ref = h5.read(golden("planet_earth_g5L20.h5"))
    assert set(ref) <= set(d), set(ref) - set(d)


def test_reader_rejects_what_it_does_not_read(tmp_path):
    """Files that are not HDF5, or of a layout outside the one the reference writes, fail with
    H5FormatError instead of returning wrong data."""
    bad = tmp_path / "x.h5"
    bad.write_bytes(b"not an hdf5 file at all" * 8)
    with pytest.raises(h5.H5FormatError):
        h5.read(str(bad))
    data = bytearray(open(golden("planet_earth_hs_g4L32.h5"), "rb").read())
    v2 = bytearray(data)
    v2[8] = 2                                  # a version-2 superblock
    (tmp_path / "v2.h5").write_bytes(bytes(v2))
    with pytest.raises(h5.H5FormatError):
        h5.read(str(tmp_path / "v2.h5"))
    sizes = bytearray(data)
    sizes[13] = 4                              # 4-byte offsets
    (tmp_path / "s4.h5").write_bytes(bytes(sizes))
    with pytest.raises(h5.H5FormatError):
        h5.read(str(tmp_path / "s4.h5"))
