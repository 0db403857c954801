"""The reference's MAT-file formats (CPU): round trips of line<is>.mat,
s_r(_).mat, s_i_r_d_std.mat and ky_w.mat through scipy.io in the reference's
layouts, the shot indices of w_load.m, and a clear error for v7.3 files."""
import numpy as np
import pytest

from gerjoii_b200 import matio, synth


def test_radargram_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    nt, nr = 50, 4
    d = rng.standard_normal((nt, nr))
    r = np.column_stack([0.5 + 0.25 * np.arange(nr), np.zeros(nr)])
    s = np.array([0.1, 0.0])
    p = str(tmp_path / "line1.mat")
    matio.save_radargram(p, d, np.arange(nt) * 1e-10, 1e-10, 2.5e8, 0.02, r, s, np.sin(np.arange(nt)))
    rg = matio.load_radargram(p)
    assert np.array_equal(rg["d"], d)
    assert rg["dt"] == 1e-10 and rg["fo"] == 2.5e8
    assert rg["dr"] == 0.25 and rg["dsr"] == pytest.approx(0.4)  # w_natur_.m:56-57
    assert rg["std_"].shape == (nt * nr, 1) and np.all(rg["std_"] == 1)


def test_s_r_indices_map_to_the_shots_of_w_load(tmp_path):
    """w_load.m:31-35: source [iz ix] -> Ez(pis + air + iz, pjs + ix) (1-based),
    receivers [ix iz] -> (pis + air + iz, pjs + ix) through w_M."""
    p = synth.small(m=20, n=30, pml=6, nt=40, free_top=True, seed=3)
    g = p.grid
    pairs = [(np.array([1, 5]), np.array([[3, 1], [7, 1], [11, 2]])),
             (np.array([2, 9]), np.array([[4, 0], [8, 0]]))]
    path = str(tmp_path / "s_r_.mat")
    matio.save_s_r(path, pairs, indexed=True)
    back = matio.load_s_r(path)
    assert all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(pairs, back))
    wv = np.random.default_rng(2).standard_normal((g.nt, 2))
    shots = matio.shots_from_s_r_(g, back, wv)
    for k, (s, r) in enumerate(pairs):
        assert (shots[k].src_i, shots[k].src_j) == (g.dom_i0 + s[0], g.dom_j0 + s[1])
        assert list(shots[k].rec) == [g.node(g.dom_i0 + iz, g.dom_j0 + ix) for ix, iz in r]
        assert np.array_equal(shots[k].wavelet, wv[:, k])


def test_dc_survey_and_ky_w_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    gathers = [{"ab": np.array([3, 5]), "current": 0.5, "mn": np.array([[7, 9], [9, 11], [11, 13]]),
                "d": rng.standard_normal(3), "std": np.full(3, 0.02)},
               {"ab": np.array([4, 8]), "current": 1.0, "mn": np.array([[12, 16]]),
                "d": rng.standard_normal(1), "std": np.full(1, 0.05)}]
    p = str(tmp_path / "s_i_r_d_std.mat")
    matio.save_dc_survey(p, gathers)
    back = matio.load_dc_survey(p)
    for a, b in zip(gathers, back):
        assert np.array_equal(a["ab"], b["ab"]) and a["current"] == b["current"]
        assert np.array_equal(a["mn"], b["mn"])
        assert np.array_equal(a["d"], b["d"]) and np.array_equal(a["std"], b["std"])
    kw = rng.random((6, 2, 2))
    q = str(tmp_path / "ky_w.mat")
    matio.save_ky_w(q, kw)
    assert np.array_equal(matio.load_ky_w(q), kw)
    matio.save_ky_w(q, kw[:, :, 0])
    assert matio.load_ky_w(q).shape == (6, 2, 1)


def test_v73_files_are_rejected_with_a_clear_error(tmp_path):
    p = tmp_path / "line1.mat"
    hdr = b"MATLAB 7.3 MAT-file, Platform: GLNXA64, Created on: Mon Jan  1 00:00:00 2024 HDF5 schema 1.00 ."
    p.write_bytes(hdr.ljust(116, b" ") + b"\x00" * 8 + b"\x00\x02" + b"IM" + b"\x00" * 512)
    with pytest.raises(ValueError, match="v7.3"):
        matio.load_radargram(str(p))


def test_dc_survey_files_to_sources(tmp_path):
    """s_i_r_d_std.mat + ky_w.mat + an electrode table -> DcSource list as
    dc_load2_5d.m and dc_electrodes.m assemble it: binning to the nearest grid
    coordinate (ties to the lower index), Robin shift, parity clean of the
    source pair only, vectorised nodes l + n (h - 1), data into d_obs."""
    from gerjoii_b200 import dc
    X = np.arange(40) * 0.25
    Z = np.arange(12) * 0.25
    robin = 1
    n, m = 40 + 2 * robin, 12 + robin
    elec = np.column_stack([0.25 * np.arange(2, 38, 2) + 0.01, np.zeros(18)])  # just off the grid points
    assert list(dc.binning(X, [0.125, 0.126, 0.124, -1.0, 99.0])) == [1, 2, 1, 1, 40]
    gathers = [{"ab": np.array([3, 5]), "current": 0.7, "mn": np.array([[7, 8], [9, 10]]),
                "d": np.array([0.1, 0.05]), "std": np.array([0.01, 0.01])}]
    kw = np.column_stack([np.geomspace(1e-3, 0.5, 6), np.ones(6)])
    matio.save_dc_survey(str(tmp_path / "s.mat"), gathers)
    matio.save_ky_w(str(tmp_path / "k.mat"), kw)
    srcs = dc.sources_from_survey(matio.load_dc_survey(str(tmp_path / "s.mat")), matio.load_ky_w(str(tmp_path / "k.mat")),
                                  X, Z, elec, robin, n, m, -0.25, 0.25)
    q = srcs[0]
    # electrode 3 sits at x = 1.51 -> grid index 7 (1-based), +1 Robin -> 8, even: kept
    # electrode 5 sits at x = 2.51 -> 11, +1 -> 12, even -> 13 (the -I electrode goes odd)
    assert (q.a, q.b) == (8 - 1, 13 - 1)
    # receivers are not cleaned: electrode k -> padded lateral 2k + 2 (1-based) -> node 2k + 1
    assert q.mn.tolist() == [[15, 17], [19, 21]]
    assert q.current == 0.7 and np.array_equal(q.d_obs, [0.1, 0.05])
    assert q.ky_w.shape == (6, 2) and q.alpha.shape == (6, dc.nalpha(n, m))


def test_radar_survey_round_trip_through_the_files(tmp_path, oracle):
    """A survey written as the reference writes it (s_r_.mat indices relative to
    the model, one line<k>.mat per shot) and read back gives the same shots,
    and the forward run of those shots reproduces the stored traces."""
    p = synth.small(m=20, n=30, pml=6, nt=120, free_top=True, seed=4)
    g = p.grid
    pairs = []
    for k, sh in enumerate(p.shots):
        iz, ix = sh.src_i - g.dom_i0, sh.src_j - g.dom_j0
        rows, cols = sh.rec % (g.NX + 1), sh.rec // (g.NX + 1)
        pairs.append((np.array([iz, ix]), np.column_stack([cols - g.dom_j0, rows - g.dom_i0])))
        d, _, _ = oracle.forward(g, p.eps_true, p.sig_true, sh)
        r = np.column_stack([(cols - g.dom_j0) * g.dx, (rows - g.dom_i0) * g.dx])
        matio.save_radargram(str(tmp_path / f"line{k + 1}.mat"), d, np.arange(g.nt) * g.dt, g.dt, 1e8, g.dx, r,
                             [ix * g.dx, iz * g.dx], sh.wavelet)
    matio.save_s_r(str(tmp_path / "s_r_.mat"), pairs, indexed=True)
    wv = np.column_stack([sh.wavelet for sh in p.shots])
    shots = matio.shots_from_s_r_(g, matio.load_s_r(str(tmp_path / "s_r_.mat")), wv)
    for k, (a, b) in enumerate(zip(p.shots, shots)):
        assert (a.src_i, a.src_j) == (b.src_i, b.src_j) and np.array_equal(a.rec, b.rec)
        d_file = matio.load_radargram(str(tmp_path / f"line{k + 1}.mat"))["d"]
        d, _, _ = oracle.forward(g, p.eps_true, p.sig_true, b)
        assert np.array_equal(d, d_file)
