"""Post-step statistics: the running sums of IO_statistics.f90 and the
plane-averaged TKE budget of tke_budget1D.f90 (one rank).

CPU tests pin the oracle's file formats and the reference behaviours it keeps
(level-1 reset of uw/vw, the cs profile read one level up, records divided by
tke_period).  GPU tests run the library on a state mirrored from the oracle
and compare: running sums exactly (both add the same FP64 products in the same
order), TKE profiles within 1e-12 (FP64) / 1e-5 (mixed) of each quantity's
scale, and the files byte layout."""
import numpy as np
import pytest

from oracle import les_oracle as O
from oracle import stats_oracle as S
from tests.helpers import mirror, oracle_run, run_params


def _state(p, steps=6, seed=0):
    ops, st = oracle_run(p, steps, seed=seed)
    return ops, st


# --------------------------------------------------------------------- CPU
def test_oracle_running_sums_cycle(tmp_path):
    p = O.Params(nx=16, ny=16, nz=8)
    ops, st = _state(p, 3)
    rs = S.RunningStats(p)
    out = str(tmp_path) + "/"
    assert not S.stat_averages(rs, st, 1, 5, 0, 4, out)
    assert S.stat_averages(rs, st, 2, 8, 0, 4, out)  # jt_total 8: written and restarted
    info = (tmp_path / "RAV_000000008_info.txt").read_text()
    assert info == f"{16:6d}{16:6d}{8:6d}{2:10d}\n"
    d3 = np.fromfile(tmp_path / "RAV_000000008_3D.dat", dtype="<f8").reshape(26, 8, 16, 16)
    np.testing.assert_array_equal(d3[0], 2 * st.u[1:9])
    np.testing.assert_array_equal(d3[S.STAT_NAMES.index("uw")][0], 0.0)
    np.testing.assert_array_equal(d3[S.STAT_NAMES.index("cs")], 2 * np.sqrt(st.cs_opt2[1:9]))
    d2 = np.fromfile(tmp_path / "RAV_000000008_2D.dat", dtype="<f8").reshape(16, 16)
    np.testing.assert_array_equal(d2, 2 * st.u_star_avg)
    assert rs.iterations == 0 and not rs.sums.any() and not rs.ustar.any()
    # not past start_stats: nothing written even on the period
    assert not S.stat_averages(rs, st, 3, 12, 12, 4, out)


# The reference's own reader of these files (matlab_src/load2decomp_RAV.m with
# the field list of matlab_src/get_data_struct_RAV.m:13-17), restated: the
# info file is four whitespace-separated integers, the 3D file the fields one
# after the other as nx*ny*nz doubles in Fortran order, the 2D file u* as
# nx*ny doubles; means are the sums over all files divided by the summed
# iteration counts.
RAV_READER_3D = ("u", "v", "w", "p", "u2", "v2", "w2", "u3", "v3", "w3", "u4", "v4", "w4",
                 "uv", "uw", "vw", "txx", "tyy", "tzz", "txy", "txz", "tyz", "dudz", "dvdz", "nut", "cs")


def _read_rav(folder, steps, nx, ny, nz):
    sums3, sums2, nt = None, None, 0
    for jt in steps:
        info = [int(x) for x in (folder / f"RAV_{jt:09d}_info.txt").read_text().split()]
        assert info[:3] == [nx, ny, nz]
        nt += info[3]
        raw = np.fromfile(folder / f"RAV_{jt:09d}_3D.dat", dtype="<f8")
        assert raw.size == len(RAV_READER_3D) * nx * ny * nz
        d3 = {n: raw[q * nx * ny * nz:(q + 1) * nx * ny * nz].reshape((nx, ny, nz), order="F")
              for q, n in enumerate(RAV_READER_3D)}
        d2 = np.fromfile(folder / f"RAV_{jt:09d}_2D.dat", dtype="<f8").reshape((nx, ny), order="F")
        sums3 = d3 if sums3 is None else {n: sums3[n] + d3[n] for n in d3}
        sums2 = d2 if sums2 is None else sums2 + d2
    return {n: v / nt for n, v in sums3.items()}, sums2 / nt, nt


def test_rav_files_follow_the_reference_reader(tmp_path):
    assert S.STAT_NAMES == RAV_READER_3D
    p = O.Params(nx=16, ny=8, nz=4)
    ops, st = _state(p, 3)
    rs = S.RunningStats(p)
    out = str(tmp_path) + "/"
    us, ws = [], []
    for jt in range(1, 7):  # two files: RAV_3 (3 iterations) and RAV_6 (3 iterations)
        st.u = st.u * 1.01  # a changing state
        st.w = st.w + 0.001
        us.append(st.u[1:p.nz + 1].copy())
        ws.append(st.w[1:p.nz + 1].copy())
        S.stat_averages(rs, st, jt, jt, 0, 3, out)
    mean3, mean2, nt = _read_rav(tmp_path, (3, 6), p.nx, p.ny, p.nz)
    assert nt == 6
    # the reader's (x, y, z) arrays are the transposes of the oracle's (z, y, x)
    np.testing.assert_allclose(mean3["u"], np.mean(us, axis=0).transpose(2, 1, 0), rtol=1e-14)
    np.testing.assert_allclose(mean3["w2"], np.mean([w * w for w in ws], axis=0).transpose(2, 1, 0), rtol=1e-14)
    np.testing.assert_allclose(mean2, st.u_star_avg.T, rtol=1e-14)


def test_oracle_tke_quirks(tmp_path):
    p = O.Params(nx=16, ny=16, nz=8)
    ops, st = _state(p, 3)
    st.cs_opt2[1:10] = np.arange(1, 10)[:, None, None] * 0.01
    means, scale = S.tke_profiles(ops, st, True)
    cs = means[S.TKE_NAMES.index("cs")]
    np.testing.assert_allclose(cs, np.arange(2, 10) * 0.01, rtol=1e-15)  # level k reads cs_opt2(k+1)
    # the plane means of spectral x, y derivatives vanish
    for n in ("dpdx", "dpdy"):
        assert np.abs(means[S.TKE_NAMES.index(n)]).max() <= 1e-12 * scale[S.TKE_NAMES.index(n)]
    # the mean of the filtered cleaned pressure is the mean of the unfiltered one
    c = st.p[1:9] - 0.5 * (st.u[1:9] ** 2 + st.v[1:9] ** 2 + (0.5 * (st.w[1:9] + st.w[2:10])) ** 2)
    np.testing.assert_allclose(means[S.TKE_NAMES.index("p")], c.mean(axis=(1, 2)), rtol=1e-12, atol=1e-14)
    # interior dpdz is the centred difference of the plane means
    mc = np.concatenate([[st.cs_opt2[1].mean()], c.mean(axis=(1, 2)), [0.0]])
    dpdz = (mc[2:] - mc[:-2]) / (2 * p.dz)
    np.testing.assert_allclose(means[S.TKE_NAMES.index("dpdz")], dpdz, rtol=1e-9, atol=1e-9 * np.abs(dpdz).max())
    # records: avar / tke_period at (ii-1)*8*nz, written when mod(jt, period) == 0
    out = str(tmp_path) + "/"
    tb = S.TkeBudget(p, out)
    assert not S.compute_tke_budget(tb, ops, st, 1, 2, True)
    assert S.compute_tke_budget(tb, ops, st, 2, 2, True)
    assert S.compute_tke_budget(tb, ops, st, 4, 2, True)  # one step summed, still divided by 2
    rec = np.fromfile(tmp_path / "ta1_profiles" / "u.out", dtype="<f8").reshape(2, 8)
    np.testing.assert_allclose(rec[0], means[0], rtol=1e-15)
    np.testing.assert_allclose(rec[1], 0.5 * means[0], rtol=1e-15)
    assert tb.ii == 3


def test_output_namelist_keys(tmp_path):
    from new_repo_b200.les import read_namelist

    f = tmp_path / "parameters.nlst"
    f.write_text("&output_param\n out_path='./out/', stat_flag=.true., start_stats=10, running_period=50,\n"
                 " tke_flag=.true., start_tke=5, tke_period=20, checkpoint=1000, scheckpoint=100 /\n")
    rp, _ = read_namelist(f)
    assert (rp.out_path, rp.stat_flag, rp.start_stats, rp.running_period) == ("./out/", True, 10, 50)
    assert (rp.tke_flag, rp.start_tke, rp.tke_period) == (True, 5, 20)


# --------------------------------------------------------------------- GPU
def _les(p, precision, **kw):
    from new_repo_b200 import LES

    return LES(run_params(p).with_(**kw), precision=precision)


def _downloaded_state(les, p):
    """An oracle State holding exactly the library's (possibly FP32) state."""
    st = O.State(p)
    for n in O.FIELDS:
        setattr(st, n, les.download(n))
    for n in ("u_star_avg",):
        setattr(st, n, les.download_plane(n))
    return st


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_running_sums_match_the_oracle_exactly(gpu, tmp_path, precision):
    p = O.Params(nx=32, ny=16, nz=8)
    _, st0 = _state(p, 6)
    gdir, odir = tmp_path / "gpu", tmp_path / "ora"
    gdir.mkdir()
    odir.mkdir()
    les = _les(p, precision, out_path=str(gdir) + "/", start_stats=4, running_period=3)
    mirror(les, st0)
    les.stat_init()
    st = _downloaded_state(les, p)
    rs = S.RunningStats(p)
    for jt_total in (4, 5, 6):  # written at 6 (running_period 3, start_stats 4)
        les.stat_averages(jt_total, jt_total)
        S.stat_averages(rs, st, jt_total, jt_total, 4, 3, str(odir) + "/")
    for suffix in ("_info.txt", "_2D.dat", "_3D.dat"):
        a = (gdir / f"RAV_000000006{suffix}").read_bytes()
        b = (odir / f"RAV_000000006{suffix}").read_bytes()
        assert a == b, suffix
    les.stat_averages(7, 7)
    S.stat_averages(rs, st, 7, 7, 4, 3, None)
    for qi, n in enumerate(S.STAT_NAMES):
        np.testing.assert_array_equal(les.stat_sums(n), rs.sums[qi], err_msg=n)
    np.testing.assert_array_equal(les.stat_sums("ustar"), rs.ustar)
    assert les.stat_iterations() == rs.iterations == 1
    les.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
@pytest.mark.parametrize("wall", [True, False])
def test_tke_budget_matches_the_oracle(gpu, tmp_path, precision, tol, wall):
    p = O.Params(nx=32, ny=32, nz=16)
    ops, st0 = _state(p, 6, seed=3)
    gdir, odir = tmp_path / "gpu", tmp_path / "ora"
    gdir.mkdir()
    odir.mkdir()
    les = _les(p, precision, out_path=str(gdir) + "/", tke_period=2,
               lbc_special="wall_law" if wall else "std")
    mirror(les, st0)
    les.tke_init()
    st = _downloaded_state(les, p)
    tb = S.TkeBudget(p, str(odir) + "/")
    for jt in (1, 2, 3):
        les.tke_budget(jt)
        S.compute_tke_budget(tb, ops, st, jt, 2, wall)
    _, scale = S.tke_profiles(ops, st, wall)
    scale = np.maximum(scale, 1e-300)
    got, rec = les.tke_profiles()
    assert rec == tb.ii == 2
    err = (np.abs(got - tb.avar).max(axis=1) / scale)
    worst = int(err.argmax())
    assert err.max() <= tol, (S.TKE_NAMES[worst], err.max())
    for qi, n in enumerate(S.TKE_NAMES):
        a = np.fromfile(gdir / "ta1_profiles" / f"{n}.out", dtype="<f8")
        b = np.fromfile(odir / "ta1_profiles" / f"{n}.out", dtype="<f8")
        assert a.shape == b.shape == (p.nz,), n
        assert np.abs(a - b).max() <= tol * scale[qi], n
    les.close()


@pytest.mark.gpu
def test_step_runs_the_statistics_its_flags_ask_for(gpu, tmp_path):
    from new_repo_b200 import log_law_noise

    p = O.Params(nx=32, ny=32, nz=16)
    les = _les(p, "fp64", out_path=str(tmp_path) + "/", stat_flag=True, start_stats=1, running_period=2,
               tke_flag=True, start_tke=0, tke_period=2)
    les.set_initial_conditions(*log_law_noise(les.params, seed=1))
    odir = tmp_path / "ora"
    odir.mkdir()
    rs = S.RunningStats(p)
    ops = O.Ops(p)
    tb = S.TkeBudget(p, str(odir) + "/")
    for _ in range(4):
        les.step(1)
        st = _downloaded_state(les, p)
        if les.jt_total > 1:
            S.stat_averages(rs, st, les.jt, les.jt_total, 1, 2, str(odir) + "/")
        S.compute_tke_budget(tb, ops, st, les.jt, 2, True)
    _, scale = S.tke_profiles(ops, st, True)
    assert sorted(f.name for f in tmp_path.glob("RAV_*")) == [
        "RAV_000000002_2D.dat", "RAV_000000002_3D.dat", "RAV_000000002_info.txt",
        "RAV_000000004_2D.dat", "RAV_000000004_3D.dat", "RAV_000000004_info.txt"]
    assert (tmp_path / "RAV_000000004_info.txt").read_text() == f"{32:6d}{32:6d}{16:6d}{2:10d}\n"
    d3 = np.fromfile(tmp_path / "RAV_000000004_3D.dat", dtype="<f8").reshape(26, 16, 32, 32)
    assert not les.stat_sums("u").any()  # restarted after the write
    assert np.isfinite(d3).all()
    for name in ("RAV_000000002_3D.dat", "RAV_000000004_3D.dat", "RAV_000000004_2D.dat"):
        assert (tmp_path / name).read_bytes() == (odir / name).read_bytes(), name
    for qi, n in enumerate(S.TKE_NAMES):
        a = np.fromfile(tmp_path / "ta1_profiles" / f"{n}.out", dtype="<f8")
        b = np.fromfile(odir / "ta1_profiles" / f"{n}.out", dtype="<f8")
        assert a.shape == b.shape == (2 * 16,), n
        assert np.abs(a - b).max() <= 1e-12 * max(scale[qi], 1e-300), n
    assert les.tke_profiles()[1] == tb.ii == 3
    les.close()


@pytest.mark.gpu
def test_spectra_windows(gpu, tmp_path):
    p = O.Params(nx=16, ny=16, nz=8)
    _, st0 = _state(p, 2)
    les = _les(p, "fp64", out_path=str(tmp_path) + "/")
    mirror(les, st0)
    les.stat_spectra(10, 1499990)  # before the first window: nothing
    les.stat_spectra(11, 1500001)  # inside, but jt not a multiple of 10
    assert not list(tmp_path.glob("SP_*"))
    les.stat_spectra(20, 1500010)
    d = np.fromfile(tmp_path / "SP_001500010.dat", dtype="<f8").reshape(3, 8, 16, 16)
    for q, n in enumerate("uvw"):
        np.testing.assert_array_equal(d[q], getattr(st0, n)[1:9])
    assert S.spectra_due(20, 1500010) and not S.spectra_due(11, 1500001)
    les.close()


@pytest.mark.gpu
def test_statistics_errors(gpu):
    from new_repo_b200 import LesError

    p = O.Params(nx=16, ny=16, nz=8)
    les = _les(p, "fp64")
    with pytest.raises(LesError) as e:
        les.stat_averages(1, 1)
    assert e.value.code == 1
    with pytest.raises(LesError) as e:
        les.tke_budget(1)
    assert e.value.code == 1
    les.params.out_path = "/nonexistent-dir/"
    les.stat_init()
    les.params.running_period = 1
    with pytest.raises(LesError) as e:
        les.stat_averages(1, 1)
    assert e.value.code == 22
    les.close()
