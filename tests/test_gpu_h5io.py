"""The field checkpoint file uvwp_NNNN.h5 through the library on the GPU.

save_4fields_fou_hdf5 (src/readwrite_hdf5.f90:276-386 with h5dump_parallel
:650-722 and writeheader_hdf5 :851-920): the library's file must equal the
oracle's restatement byte for byte, and the oracle's independent reader must
decode it to the device fields bit for bit.  read_4fields_fou_hdf5 (:5-197):
the library reads its own and the oracle's files back bit for bit, drops or
zero-fills modes as the reference does and refuses another y-z resolution.
The stepper writes its state and restarts from it (src/main1.f90:735-752):
a restarted run repeats the original bit for bit.
"""
import numpy as np
import pytest

import duct_b200 as D
from duct_b200 import synth
from oracle import h5file as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with D.Context(0) as c:
        yield c


def fields(my, mz, nm, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.standard_normal((my, mz, nm)) + 1j * rng.standard_normal((my, mz, nm)))
            for _ in range(4)]


def dev(ctx, a):
    d = ctx.device_array(a.shape)
    d.upload(a)
    return d


def header(my, mz, nm, **kw):
    h = dict(numerop=1, mgalx=3 * nm, my=my, mz=mz, mx1=nm - 1, alp=0.5, aspect=1.0, time=1.25, fnu=1 / 4400.0,
             cfl=0.0, dtfixed=2e-4, cmassflow=1.9, slip=0.0, divergence=1e-13)
    h.update(kw)
    return h


# (33, 33, 11): one chunk per field; (129, 129, 43): 11.4 MB fields, two
# 8 MiB staging chunks each (the double-buffered path); (17, 9, 3): my != mz
@pytest.mark.parametrize("my,mz,nm", [(33, 33, 11), (129, 129, 43), (17, 9, 3)])
def test_save_equals_oracle_file_and_decodes(ctx, tmp_path, my, mz, nm):
    host = fields(my, mz, nm, my + nm)
    d = [dev(ctx, f) for f in host]
    hdr = header(my, mz, nm)
    path = tmp_path / "uvwp_0003.h5"
    try:
        ctx.save_4fields_fou_hdf5_dev(str(path), *d, hdr)
        buf = path.read_bytes()
        ref = H.write_4fields(host, hdr)
        assert len(buf) == len(ref)
        diff = np.flatnonzero(np.frombuffer(buf, np.uint8) != np.frombuffer(ref, np.uint8))
        assert diff.size == 0, "first differing byte at %d of %d" % (diff[0], len(buf))
        ds = H.read(buf)
        for a, b in zip(H.fields_of(ds), host):
            assert np.array_equal(a, b)
        h = H.header_of(ds)
        for k, v in hdr.items():
            assert h[k] == v, k
        # read back through the library into fresh device fields
        back = [ctx.device_array((my, mz, nm)) for _ in range(4)]
        got_hdr = ctx.read_4fields_fou_hdf5_dev(str(path), *back)
        for a, b in zip(back, host):
            assert np.array_equal(a.download(), b)
            a.free()
        for k, v in hdr.items():
            assert got_hdr[k] == v, k
    finally:
        for a in d:
            a.free()


def test_read_oracle_file_with_fewer_and_more_modes(ctx, tmp_path):
    """h5load_parallel + the copy of read_4fields_fou_hdf5: modes beyond the
    run's are dropped, missing ones are zero."""
    my, nm = 33, 11
    host = fields(my, my, nm, 5)
    path = tmp_path / "f.h5"
    path.write_bytes(H.write_4fields(host, header(my, my, nm)))
    for want in (7, 11, 15):
        out = [ctx.device_array((my, my, want)) for _ in range(4)]
        try:
            for a in out:
                a.upload(np.full((my, my, want), 7.0 + 7.0j))
            ctx.read_4fields_fou_hdf5_dev(str(path), *out)
            for a, b in zip(out, host):
                g = a.download()
                k = min(want, nm)
                assert np.array_equal(g[:, :, :k], b[:, :, :k])
                assert not np.any(g[:, :, k:])
        finally:
            for a in out:
                a.free()


def test_read_refuses_an_old_grid_the_transform_cannot_take(ctx, tmp_path):
    """my - 1 = 7^2: no Chebyshev transform of the old planes -- refused
    before the fields are touched."""
    host = fields(50, 50, 3, 9)
    path = tmp_path / "odd.h5"
    path.write_bytes(H.write_4fields(host, header(50, 50, 3)))
    out = [ctx.device_array((33, 33, 3)) for _ in range(4)]
    try:
        for a in out:
            a.upload(np.full((33, 33, 3), 2.0 + 1.0j))
        with pytest.raises(D.DuctGPUError, match="re-interpolated"):
            ctx.read_4fields_fou_hdf5_dev(str(path), *out)
        assert np.all(out[0].download() == 2.0 + 1.0j)      # untouched
    finally:
        for a in out:
            a.free()


def test_read_refuses_one_changed_size_and_host_fields(ctx, tmp_path):
    my, nm = 33, 5
    host = fields(my, my, nm, 6)
    path = tmp_path / "f.h5"
    path.write_bytes(H.write_4fields(host, header(my, my, nm)))
    out = [ctx.device_array((65, 33, nm)) for _ in range(4)]
    try:
        before = out[0].download()
        with pytest.raises(D.DuctGPUError, match="re-interpolate"):
            ctx.read_4fields_fou_hdf5_dev(str(path), *out)
        assert np.array_equal(out[0].download(), before)    # nothing written
    finally:
        for a in out:
            a.free()
    d = [dev(ctx, f) for f in host]
    try:
        with pytest.raises(D.DuctGPUError, match="device memory"):
            ctx.save_4fields_fou_hdf5_dev(str(tmp_path / "g.h5"), host[0].ctypes.data, *d[1:], header(my, my, nm))
        with pytest.raises(D.DuctGPUError):
            ctx.save_4fields_fou_hdf5_dev(str(tmp_path / "no/such/dir/g.h5"), *d, header(my, my, nm))
    finally:
        for a in d:
            a.free()


def test_dns_save_and_restart_repeat_the_run(ctx, tmp_path):
    m, mgalx, alp, fnu, dt = 33, 64, 1.0, 1.0 / 2000.0, 1e-3
    u, v, w, p, dpval = synth.dns_initial(mgalx, m, alp, 0.1, seed=11)
    ctx.pseudomat(m, m)
    path = str(tmp_path / D.uvwp_filename("", 1))
    with D.Dns(ctx, mgalx, alp, fnu, dt, cmassflow=True) as dns:
        dns.set_fields(u, v, w, p)
        dns.steps(2)
        dns.save_hdf5(path, time=2 * dt, cfl=0.25)
        saved = dns.fields()
        divmax = dns.statistics()["divmax"]
        slip = dns.cfl()["slip"]
        dns.steps(2)
        after = dns.fields()
    ds = H.read(open(path, "rb").read())
    for a, b in zip(H.fields_of(ds), saved):
        assert np.array_equal(a, b)
    h = H.header_of(ds)
    assert (h["mgalx"], h["my"], h["mz"], h["mx1"]) == (mgalx, m, m, saved[0].shape[2] - 1)
    assert h["dtfixed"] == dt and h["time"] == 2 * dt and h["cfl"] == 0.25 and h["alp"] == alp
    assert h["divergence"] == divmax[2]
    assert h["slip"] == slip            # the measured wall slip of the last step
    # the restart holds the file's cmassflow, the run's own flow rate: the
    # run repeats bit for bit
    with D.Dns(ctx, mgalx, alp, fnu, dt, cmassflow=True) as dns:
        assert dns.load_hdf5(path) == 2 * dt
        for a, b in zip(dns.fields(), saved):
            assert np.array_equal(a, b)
        dns.steps(2)
        for a, b in zip(dns.fields(), after):
            assert np.array_equal(a, b)


def test_dns_statistics_file_equals_oracle_file(ctx, tmp_path):
    """write_statistics_hdf5 (src/readwrite_hdf5.f90:388-648): the stepper's
    file equals the oracle's restatement of it, byte for byte, for the same
    accumulated statistics."""
    m, mgalx, alp, fnu, dt = 33, 64, 1.0, 1.0 / 2000.0, 1e-3
    u, v, w, p, _ = synth.dns_initial(mgalx, m, alp, 0.1, seed=12)
    ctx.pseudomat(m, m)
    path = D.statistics_filename(str(tmp_path) + "/")
    with D.Dns(ctx, mgalx, alp, fnu, dt, cmassflow=True) as dns:
        dns.set_fields(u, v, w, p)
        dns.steps(3, stats_every=1)
        dns.write_statistics_hdf5(path, time=3 * dt, timef=0.0)
        st = dns.statistics()
        om = dns.statistics_omg()
    assert path.endswith("statistics_0001.h5")
    ref = H.write_statistics(dict(mgalx=mgalx, my=m, mz=m, nstat=st["nstat"], timef=0.0, time=3 * dt, fnu=fnu,
                                  alp=alp, aspect=1.0, mean=st["mean"], prod=st["prod"], ppb=st["ppb"],
                                  spec=st["spec"], om2=om["om2"]))
    buf = open(path, "rb").read()
    assert buf == ref
    ds = H.read(buf)
    assert int(ds["nstat"][0]) == 3 and np.array_equal(ds["ox2"], om["om2"][0].T)



@pytest.mark.parametrize("src,dst,nm", [((65, 65), (97, 129), 6), ((129, 97), (33, 65), 4)])
def test_read_reinterpolates_another_grid(ctx, oracle, tmp_path, src, dst, nm):
    """read_4fields_fou_hdf5 with cheb_interp (src/chebyshev.f90:725-765):
    against the oracle's restatement, and exact for fields that are
    polynomials of degree < 20 in y and z."""
    (myr, mzr), (my, mz) = src, dst
    rng = np.random.default_rng(myr + my)
    # polynomials of degree 12 in y and 9 in z at the old nodes (complex,
    # every mode) -- cheb_interp reproduces them at the new nodes
    yr, zr = -np.cos(np.arange(myr) * np.pi / (myr - 1)), -np.cos(np.arange(mzr) * np.pi / (mzr - 1))
    y, z = -np.cos(np.arange(my) * np.pi / (my - 1)), -np.cos(np.arange(mz) * np.pi / (mz - 1))
    A = rng.standard_normal((13, 10, nm, 4)) + 1j * rng.standard_normal((13, 10, nm, 4))

    def poly(yy, zz):
        P = np.polynomial.polynomial
        return [np.asfortranarray(np.stack([P.polygrid2d(yy, zz, A[:, :, m, f])
                                            for m in range(nm)], axis=2)) for f in range(4)]

    host, exact = poly(yr, zr), poly(y, z)
    path = tmp_path / "old.h5"
    path.write_bytes(H.write_4fields(host, header(myr, mzr, nm)))
    out = [ctx.device_array((my, mz, nm)) for _ in range(4)]
    try:
        h = ctx.read_4fields_fou_hdf5_dev(str(path), *out)
        assert (h["my"], h["mz"]) == (myr, mzr)
        for a, f, e in zip(out, host, exact):
            g = a.download()
            ref = oracle.cheb_interp(f, my, mz)
            assert np.abs(g - ref).max() < 1e-12 * np.abs(ref).max()
            assert np.abs(g - e).max() < 1e-11 * np.abs(e).max()
    finally:
        for a in out:
            a.free()
