"""The field checkpoint file uvwp_NNNN.h5 and the statistics file
statistics_NNNN.h5 on the CPU: the oracle's writers against its independent
reader, the library's header reader and file name rules against the oracle
(no GPU: the library's HDF5 reader of the header is host code), and the
reader's refusals of damaged files.

Reference: save_4fields_fou_hdf5 / writeheader_hdf5 / readheader_hdf5 /
write_statistics_hdf5 (src/readwrite_hdf5.f90:276-386, 388-648, 799-920),
concat5b / concatb (src/concat.F:33-45, 74-87).
"""
import numpy as np
import pytest

import duct_b200 as D
from oracle import h5file as H


def fields(my, mz, nm, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(4):
        f = rng.standard_normal((my, mz, nm)) + 1j * rng.standard_normal((my, mz, nm))
        out.append(np.asfortranarray(f))
    return out


HDR = dict(numerop=1, mgalx=16, my=9, mz=7, mx1=4, alp=0.5, aspect=1.25, time=3.75, fnu=1 / 4400.0,
           cfl=0.3, dtfixed=2e-4, cmassflow=1.92783343620839, slip=1e-17, divergence=3.5e-13)


def test_oracle_writer_reader_roundtrip():
    f = fields(9, 7, 5, 1)
    buf = H.write_4fields(f, HDR)
    ds = H.read(buf)
    assert ds["u"].shape == (5, 7, 9, 2) and ds["u"].dtype == np.float64
    for a, b in zip(H.fields_of(ds), f):
        assert np.array_equal(a, b)
    h = H.header_of(ds)
    assert h["nparams"] == 7
    for k, v in HDR.items():
        assert h[k] == v, k


def test_oracle_file_layout_facts():
    """Big-endian doubles in (mx1+1, mz, my, 2) order at a 4 KiB-aligned
    offset; the file ends at the superblock's end-of-file address."""
    f = fields(9, 7, 5, 2)
    buf = H.write_4fields(f, HDR)
    eof = int.from_bytes(buf[40:48], "little")
    assert eof == len(buf)
    raw = f[0].reshape(-1, order="F").view(np.float64).astype(">f8").tobytes()
    at = buf.find(raw)
    assert at > 0 and at % 4096 == 0


def test_library_reads_oracle_header(tmp_path):
    path = tmp_path / "uvwp_0003.h5"
    path.write_bytes(H.write_4fields(fields(9, 7, 5, 3), HDR))
    h = D.read_hdf5_header(str(path))
    assert h["nparams"] == 7
    for k, v in HDR.items():
        assert h[k] == v, k


def test_library_header_without_mx1(tmp_path):
    """readheader_hdf5 (src/readwrite_hdf5.f90:822-825): a file without mx1
    holds the 2/3-rule modes of mgalx."""
    hdr = dict(HDR, mgalx=64, mx1=20)
    path = tmp_path / "old.h5"
    path.write_bytes(H.write_4fields(fields(9, 7, 21, 4), hdr, omit=("mx1", "numerop")))
    h = D.read_hdf5_header(str(path))
    assert h["mx1"] == 2 * (64 // 3) // 2 - 1 == 20
    assert h["numerop"] == 1


def test_library_reads_file_behind_a_user_block(tmp_path):
    """A superblock after a 512-byte user block: addresses count from it."""
    buf = H.write_4fields(fields(9, 7, 5, 5), HDR)
    path = tmp_path / "ub.h5"
    path.write_bytes(b"\0" * 512 + buf)
    assert D.read_hdf5_header(str(path))["time"] == HDR["time"]
    assert H.header_of(H.read(path.read_bytes()))["time"] == HDR["time"]


@pytest.mark.parametrize("cut", ["truncated", "signature", "snod", "heap", "empty", "cycle"])
def test_library_refuses_damaged_files(tmp_path, cut):
    buf = bytearray(H.write_4fields(fields(9, 7, 5, 6), HDR))
    if cut == "cycle":
        # a level-1 B-tree node whose 32 children are itself: refused (a
        # bound on the nodes visited), not walked 32^16 times
        at = buf.find(b"TREE")
        buf[at + 4:at + 8] = bytes([0, 1, 32, 0])
        for i in range(32):
            buf[at + 32 + 16 * i:at + 40 + 16 * i] = at.to_bytes(8, "little")
    elif cut == "truncated":
        buf = buf[:len(buf) // 2]
    elif cut == "signature":
        buf[1:4] = b"XYZ"
    elif cut == "snod":
        at = buf.find(b"SNOD")
        buf[at:at + 4] = b"SNOX"
    elif cut == "heap":
        at = buf.find(b"HEAP")
        buf[at + 8:at + 16] = (1 << 40).to_bytes(8, "little")   # heap larger than the file
    else:
        buf = bytearray()
    path = tmp_path / "bad.h5"
    path.write_bytes(bytes(buf))
    with pytest.raises(D.DuctGPUError):
        D.read_hdf5_header(str(path))
    if cut != "empty":
        with pytest.raises(H.FormatError):
            H.read(bytes(buf))


def test_library_refuses_missing_file(tmp_path):
    with pytest.raises(D.DuctGPUError):
        D.read_hdf5_header(str(tmp_path / "nothing.h5"))


@pytest.mark.parametrize("prefix,iimag", [("run/", 0), ("run/", 7), ("/data/duct_", 123), ("out ", 9999),
                                          ("a b c", 42), ("x/", 10000), ("x/", -1)])
def test_uvwp_filename_matches_concat5b(prefix, iimag):
    assert D.uvwp_filename(prefix, iimag) == H.uvwp_filename(prefix, iimag)


def test_uvwp_filename_examples():
    assert D.uvwp_filename("run/", 12) == "run/uvwp_0012.h5"
    assert D.uvwp_filename("out   ", 3) == "outuvwp_0003.h5"
    assert D.uvwp_filename("x/", 12345) == "x/uvwp_****.h5"


def test_statistics_filename_takes_the_first_free_number(tmp_path):
    """concatb(fuvwpout,'statistics_',11,ext,4,'.h5',3,filename) with the first
    icf whose file does not exist (src/readwrite_hdf5.f90:446-456)."""
    prefix = str(tmp_path) + "/"
    assert D.statistics_filename(prefix) == prefix + "statistics_0001.h5"
    (tmp_path / "statistics_0001.h5").write_bytes(b"")
    (tmp_path / "statistics_0002.h5").write_bytes(b"")
    assert D.statistics_filename(prefix + " ignored") == prefix + "statistics_0003.h5"


def test_oracle_statistics_file_decodes():
    my, mz, M = 9, 9, 4
    rng = np.random.default_rng(3)
    st = dict(mgalx=12, my=my, mz=mz, nstat=5, timef=0.5, time=2.0, fnu=1e-3, alp=0.5, aspect=1.0,
              mean=rng.standard_normal((4, my, mz)), prod=rng.standard_normal((6, my, mz)),
              ppb=rng.standard_normal((my, mz)), spec=rng.standard_normal((4, 7, M)),
              om2=rng.standard_normal((3, my, mz)))
    ds = H.read(H.write_statistics(st))
    assert np.array_equal(ds["um"], st["mean"][0].T) and np.array_equal(ds["ppst"], st["spec"][3])
    assert np.array_equal(ds["uvb"], st["prod"][3].T) and np.array_equal(ds["oz2"], st["om2"][2].T)
    assert int(ds["nstat"][0]) == 5 and list(ds["jinco"]) == [0, 1, 2, 4, 0, 1, 2]


@pytest.mark.parametrize("src,dst", [((65, 65), (97, 129)), ((129, 97), (33, 65))])
def test_oracle_cheb_interp_is_exact_for_low_degree_polynomials(oracle, src, dst):
    """cheb_interp (src/chebyshev.f90:725-765) keeps 20 x 20 Chebyshev
    coefficients: a polynomial of degree 12 in y and 9 in z at the old nodes
    comes out exactly at the new ones (pins the node and sign convention)."""
    (myr, mzr), (my, mz) = src, dst
    P = np.polynomial.polynomial
    A = np.random.default_rng(0).standard_normal((13, 10))
    nodes = lambda n: -np.cos(np.arange(n) * np.pi / (n - 1))
    f = np.asfortranarray(P.polygrid2d(nodes(myr), nodes(mzr), A)[:, :, None].astype(complex))
    e = P.polygrid2d(nodes(my), nodes(mz), A)
    g = oracle.cheb_interp(f, my, mz)[:, :, 0]
    assert np.abs(g - e).max() < 1e-13 * np.abs(e).max()


@pytest.mark.parametrize("x,want", [(1.0, " 0.10000000E+01"), (-2.5e-4, "-0.25000000E-03"), (0.0, " 0.00000000E+00"),
                                    (123456789.0, " 0.12345679E+09"), (0.999999999, " 0.10000000E+01"),
                                    (1.0e-10, " 0.10000000E-09"), (-7.0, "-0.70000000E+01")])
def test_fortran_e15_8(x, want):
    assert D.fortran_e15_8(x) == want


def test_ener_line_columns_feed_the_reference_parser():
    """utils/gen_tsd2hdf5.py:37-42 reads awk columns 14-17 of the ENER lines as
    the om_x sector energies Sn, Sw, Ss, Se."""
    hist = [1.0, 2.0, 3.0, 4.0, 0.1, 0.2, 0.3, 0.11, 0.21, 0.31]
    omg = [5.0, 6.0, 7.0, 8.0, 9.0, 10.0, 11.0, 12.0, 13.0, 14.0, 0.5, 0.6, 0.7, 0.51, 0.61, 0.71]
    line = D.ener_line(0.25, hist, omg)
    cols = line.split()
    assert cols[0] == "ENER:" and len(cols) == 39
    assert [float(c) for c in cols[13:17]] == [5.0, 6.0, 7.0, 8.0]     # awk $14..$17
    assert float(cols[1]) == 0.25 and float(cols[2]) == 10.0 and float(cols[3]) == pytest.approx(0.6)
    assert float(cols[8]) == pytest.approx(35.0 ** 0.5)                  # sqrt of the five sector energies
    assert [float(c) for c in cols[32:38]] == [0.5, 0.6, 0.7, 0.51, 0.61, 0.71]
