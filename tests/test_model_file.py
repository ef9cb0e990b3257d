"""The .saige.model writer (null_model.rs:17-113, serialization.rs:13-34): NullModel
as bincode 1.3.3 writes it (fixed-width little-endian integers, u64 lengths, u32 enum
variant index), checked against bytes built here from those rules."""
import struct

import numpy as np
import pytest

import csaige_b200 as cs


def _vec(a):
    return struct.pack("<Q", len(a)) + b"".join(struct.pack("<d", v) for v in a)


def _str(s):
    return struct.pack("<Q", len(s)) + s.encode()


def test_tiny_model_bytes(tmp_path):
    vr = cs.VarianceRatioResult(0.9, [], 3, np.array([1.0]), np.zeros(0, np.int64))
    f = tmp_path / "t.saige.model"
    cs.save_model(f, cs.TraitType.Binary, ["a", "bc"], [1.0, 0.5], [0.25], [0.5, 0.25],
                  [1.0, 0.0], np.array([[1.0], [1.0]]), [0.5, 0.5], vr)
    want = (b"SGMD" + struct.pack("<I", 1) + struct.pack("<I", 0)
            + struct.pack("<Q", 2) + _str("a") + _str("bc")
            + struct.pack("<QQ", 2, 1) + struct.pack("<dd", 1.0, 0.5)
            + _vec([0.25]) + _vec([0.5, 0.25])
            + _vec([0.25, 0.1875])            # mu2 = mu (1 - mu)
            + _vec([0.5, -0.25])              # residuals = y - mu
            + _vec([1.0, 0.0]) + _vec([1.0, 1.0]) + struct.pack("<Q", 1) + _vec([0.5, 0.5])
            + struct.pack("<d", 0.9) + struct.pack("<Q", 0) + struct.pack("<Q", 3)
            + _vec([1.0])
            + b"\x00" + struct.pack("<QQQ", 0, 0, 0) + b"\x00" + struct.pack("<Q", 0))
    assert f.read_bytes() == want


def test_round_trip_with_loco(tmp_path):
    rng = np.random.default_rng(0)
    n, p = 50, 3
    x = np.column_stack([np.ones(n), rng.standard_normal((n, p - 1))])
    mu = rng.uniform(0.05, 0.95, n)
    y = (rng.random(n) < mu).astype(float)
    w = mu * (1 - mu)
    xv = cs.xvx_inv_xv(x, w)
    vr = cs.VarianceRatioResult(1.02, [(10.5, 0.97), (float("inf"), 1.05)], 40,
                                rng.uniform(0.9, 1.1, 40), np.zeros(0, np.int64))
    loco = {c: cs.LocoChromResult(c, np.array([1.0, 0.2 + k]), mu, y - mu, w, np.zeros(p))
            for k, c in enumerate(["1", "10", "2"])}
    ids = [f"id{i}" for i in range(n)]
    f = tmp_path / "r.saige.model"
    cs.save_model(f, cs.TraitType.Binary, ids, [1.0, 0.3], [0.1, 0.2, 0.3], mu, y, x, xv, vr,
                  loco=loco, n_markers_in_grm=1234)
    m = cs.load_model(f)
    assert m.magic == b"SGMD" and m.version == 1 and m.trait_type == cs.TraitType.Binary
    assert m.sample_ids == ids and m.n_samples == n and m.n_covariates == p and m.x_ncols == p
    assert np.array_equal(m.mu, mu) and np.array_equal(m.y, y)
    assert np.array_equal(m.mu2, mu * (1 - mu)) and np.array_equal(m.residuals, y - mu)
    assert np.array_equal(m.x_flat, x.T.ravel()) and np.array_equal(m.xvx_inv_xv_flat, xv)
    assert m.variance_ratio.variance_ratio == 1.02
    assert m.variance_ratio.categorical_vr == [(10.5, 0.97), (float("inf"), 1.05)]
    assert m.use_loco and [c for c, _ in m.loco_tau] == ["1", "10", "2"]
    assert m.loco_tau[2][1] == (1.0, 2.2)
    assert np.array_equal(m.loco_mu[0][1], mu)
    assert m.n_markers_in_grm == 1234 and not m.use_sparse_grm


def test_quantitative_mu2_is_one(tmp_path):
    vr = cs.VarianceRatioResult(1.0, [], 0, np.zeros(0), np.zeros(0, np.int64))
    f = tmp_path / "q.saige.model"
    cs.save_model(f, cs.TraitType.Quantitative, ["a", "b"], [1.0, 0.5], [0.0], [0.3, 0.7],
                  [1.0, 2.0], np.ones((2, 1)), [0.5, 0.5], vr)
    m = cs.load_model(f)
    assert np.array_equal(m.mu2, [1.0, 1.0]) and m.trait_type == cs.TraitType.Quantitative


def test_bad_magic_is_rejected(tmp_path):
    vr = cs.VarianceRatioResult(1.0, [], 0, np.zeros(0), np.zeros(0, np.int64))
    f = tmp_path / "b.saige.model"
    cs.save_model(f, cs.TraitType.Binary, ["a"], [1.0, 0.5], [0.0], [0.3], [1.0], np.ones((1, 1)),
                  [1.0], vr)
    data = bytearray(f.read_bytes())
    data[0:4] = b"XXXX"
    f.write_bytes(bytes(data))
    with pytest.raises(ValueError, match="magic"):
        cs.load_model(f)


def test_xvx_inv_xv_layout():
    # fit_null.rs:294-305: data[j*n + i] = ((X'WX)^-1 X'W)[j, i]
    rng = np.random.default_rng(1)
    n, p = 40, 4
    x = rng.standard_normal((n, p))
    w = rng.uniform(0.1, 1.0, n)
    got = cs.xvx_inv_xv(x, w).reshape(p, n)
    want = np.linalg.solve(x.T @ (w[:, None] * x), x.T * w)
    assert np.allclose(got, want, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("prefix,stem", [("out/example", "out/example"),
                                         ("out/example.v1", "out/example"),
                                         ("run", "run")])
def test_output_names_follow_with_extension(prefix, stem):
    assert cs.api._with_extension(prefix, "saige.model") == stem + ".saige.model"
    assert cs.api._with_extension(prefix, "varianceRatio.txt") == stem + ".varianceRatio.txt"
