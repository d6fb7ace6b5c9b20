"""General float / half descriptors through the reference-named entry points.

The reference's own default benchmark data are unit-normalised vectors of
rand() values (src/test.cu:41,70-74, src/helper.cu:40-58), not integers; these
take the library's float path (split FP16 hi + lo rows for float input, FP16
rows in place for half input, f32 accumulation on the tensor cores, float
keys). The checker is the FP64 oracle (oracle.brute_2nn_f64).

Tolerance, stated per query and base row b: a distance may differ from the
FP64 one by at most TOL * (|q|^2 + |b|^2) with TOL = 2^-16 (the split rows
carry 22 significant bits per value and the accumulation is f32; the bound
keeps a wide margin over both). An index may differ from the oracle's only
when the FP64 distances of the two rows lie within twice that tolerance (a
swap among near-ties), for the nearest and for the second nearest.
"""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle

pytestmark = pytest.mark.gpu
TOL = 2.0 ** -16


def rand_unit(n, seed):
    """Like make_rand_vec_array: rand()-range integers, L2-normalised (all components >= 0)."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 2 ** 31 - 1, (n, 128)).astype(np.float64)
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


def gauss(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, 128)) * scale).astype(np.float32)


def _f64_dist(q, r, qi, ri, metric):
    qq = q[qi].astype(np.float64)
    rr = r[ri].astype(np.float64)
    if metric == ms.METRIC_L2:
        return ((qq - rr) ** 2).sum(-1)
    return -2.0 * (qq * rr).sum(-1)


def check_2nn(q, r, got_d, got_i, metric=ms.METRIC_L2):
    """got_d, got_i: [n, 2] GPU distances / indices (float32 / int)."""
    want_d, want_i = oracle.brute_2nn_f64(q, r, metric=metric)
    n = q.shape[0]
    rows = np.arange(n)
    qn = (q.astype(np.float64) ** 2).sum(1)
    rn = (r.astype(np.float64) ** 2).sum(1)
    swaps = 0
    for c in range(2):
        gi = got_i[:, c].astype(np.int64)
        assert (gi >= 0).all() and (gi < r.shape[0]).all()
        tol = TOL * (qn + rn[gi]) if metric == ms.METRIC_L2 else TOL * 2 * np.sqrt(qn * rn[gi])
        true_d = _f64_dist(q, r, rows, gi, metric)
        err = np.abs(got_d[:, c].astype(np.float64) - true_d)
        assert (err <= tol).all(), f"distance error {err.max()} > tol at column {c}"
        differ = gi != want_i[:, c]
        swaps += int(differ.sum())
        assert (true_d[differ] <= want_d[differ, c] + 2 * tol[differ]).all(), f"index swap beyond tolerance, column {c}"
    assert (got_i[:, 0] != got_i[:, 1]).all()
    return swaps


@pytest.mark.parametrize("data", ["rand_unit", "gauss", "gauss_large", "gauss_tiny"])
def test_float_device_search_vs_fp64(cuda_device, data):
    import torch

    gen = {"rand_unit": lambda n, s: rand_unit(n, s), "gauss": lambda n, s: gauss(n, s),
           "gauss_large": lambda n, s: gauss(n, s, 3.0e6), "gauss_tiny": lambda n, s: gauss(n, s, 1.0e-7)}[data]
    q, r = gen(700, 1), gen(9000, 2)
    out = ms.match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device), threshold=0.8,
                   outputs=("nn_idx", "nn_dist", "matches"))
    assert ms.stream_status() == ms.SIFT_OK
    check_2nn(q, r, out["nn_dist"].cpu().numpy(), out["nn_idx"].cpu().numpy())


def test_half_device_search_vs_fp64(cuda_device):
    """Half rows searched in place: exact FP16 products, f32 accumulation."""
    import torch

    q = rand_unit(600, 3).astype(np.float16)
    r = rand_unit(8000, 4).astype(np.float16)
    out = ms.match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device), threshold=0.8,
                   outputs=("nn_idx", "nn_dist"))
    assert ms.stream_status() == ms.SIFT_OK
    check_2nn(q.astype(np.float32), r.astype(np.float32), out["nn_dist"].cpu().numpy(), out["nn_idx"].cpu().numpy())


def test_reference_entry_points_on_reference_default_data(cuda_device):
    """cublas_2nn_sift (device, host and half inputs), cublas_2nn_f, device_brute
    and host_brute on the reference benchmark's own kind of data."""
    import torch

    q_n, r_n = 500, 12000
    q, r = rand_unit(q_n, 5), rand_unit(r_n, 6)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    want_d, want_i = oracle.brute_2nn_f64(q, r)

    s = torch.zeros((q_n, 4), dtype=torch.float32, device=cuda_device)
    ms.device_brute(qd, rd, q_n, r_n, s)
    got = s.cpu().numpy()
    check_2nn(q, r, got[:, :2], got[:, 2:].astype(np.int64))

    hs = np.zeros((q_n, 4), np.float32)
    ms.host_brute(q, r, q_n, r_n, hs)
    np.testing.assert_array_equal(hs, got)

    ms.cublas_2nn_f(qd, rd, q_n, r_n, s)
    got_f = s.cpu().numpy()
    check_2nn(q, r, got_f[:, :2], got_f[:, 2:].astype(np.int64), metric=ms.METRIC_DOT)

    # threshold 2 (the reference benchmark's setting, src/test.cu:210): every
    # query matches its nearest row
    m = torch.zeros(q_n, dtype=torch.int32, device=cuda_device)
    assert ms.cublas_2nn_sift(qd, rd, ms.FLOAT_DEVICE, q_n, r_n, m, 2.0) == ms.SIFT_OK
    np.testing.assert_array_equal(m.cpu().numpy(), got[:, 2].astype(np.int32))
    m_host = np.zeros(q_n, np.uint32)
    assert ms.cublas_2nn_sift(q, r, ms.FLOAT_HOST, q_n, r_n, m_host, 2.0) == ms.SIFT_OK
    np.testing.assert_array_equal(m_host.astype(np.int64), got[:, 2].astype(np.int64))
    # ratio test at 0.8 against FP64 ratios, near-threshold cases excepted
    m8 = torch.zeros(q_n, dtype=torch.int32, device=cuda_device)
    assert ms.cublas_2nn_sift(qd, rd, ms.FLOAT_DEVICE, q_n, r_n, m8, 0.8) == ms.SIFT_OK
    ratio = np.sqrt(want_d[:, 0] / want_d[:, 1])
    want_m = np.where(ratio < 0.8, want_i[:, 0], 0xFFFFFFFF).astype(np.uint32)
    got_m = m8.cpu().numpy().view(np.uint32)
    near = np.abs(ratio - 0.8) < 1e-3
    np.testing.assert_array_equal(got_m[~near], want_m[~near])
    # half input: same search on the rows rounded to FP16
    qh, rh = qd.half(), rd.half()
    mh = torch.zeros(q_n, dtype=torch.int32, device=cuda_device)
    assert ms.cublas_2nn_sift(qh, rh, ms.HALF_DEVICE, q_n, r_n, mh, 2.0) == ms.SIFT_OK
    sh = torch.zeros((q_n, 4), dtype=torch.float32, device=cuda_device)
    out = ms.match(qh, rh, threshold=2.0, outputs=("nn_idx", "nn_dist"))
    check_2nn(qh.float().cpu().numpy(), rh.float().cpu().numpy(), out["nn_dist"].cpu().numpy(),
              out["nn_idx"].cpu().numpy())
    np.testing.assert_array_equal(mh.cpu().numpy(), out["nn_idx"][:, 0].cpu().numpy())
    del sh


def test_float_path_against_reference_device_brute(cuda_device):
    """The reference's own device_brute (FP32 SIMT, built from its sources) on
    the same rand() data: distances agree within the tolerance, indices agree
    except for near-ties."""
    import torch

    if not oracle.ref_available():
        pytest.skip("reference library not built")
    q_n, r_n = 300, 6000
    q, r = rand_unit(q_n, 7), rand_unit(r_n, 8)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    s_ref = torch.zeros((q_n, 4), dtype=torch.float32, device=cuda_device)
    assert oracle.ref().ref_device_brute(qd.data_ptr(), rd.data_ptr(), q_n, r_n, s_ref.data_ptr()) == 0
    ref = s_ref.cpu().numpy()
    s = torch.zeros((q_n, 4), dtype=torch.float32, device=cuda_device)
    ms.device_brute(qd, rd, q_n, r_n, s)
    got = s.cpu().numpy()
    check_2nn(q, r, got[:, :2], got[:, 2:].astype(np.int64))
    qn = (q.astype(np.float64) ** 2).sum(1)
    for c in range(2):
        rn = (r[got[:, 2 + c].astype(np.int64)].astype(np.float64) ** 2).sum(1)
        assert (np.abs(got[:, c] - ref[:, c]) <= 2 * TOL * (qn + rn)).all()


@pytest.mark.parametrize("bad", ["nan", "inf"])
def test_non_finite_values_are_rejected(cuda_device, bad):
    import torch

    q, r = rand_unit(20, 9), rand_unit(100, 10)
    q[3, 7] = np.nan if bad == "nan" else np.inf
    for dt, typ in ((torch.float32, ms.FLOAT_DEVICE), (torch.float16, ms.HALF_DEVICE)):
        m = torch.zeros(20, dtype=torch.int32, device=cuda_device)
        rc = ms.cublas_2nn_sift(torch.from_numpy(q).to(cuda_device).to(dt), torch.from_numpy(r).to(cuda_device).to(dt),
                                typ, 20, 100, m, 0.8)
        assert rc == ms.SIFT_ERR_INVALID_ARG, (dt, rc)


def test_integer_data_still_takes_the_exact_path(cuda_device):
    """Integer-valued floats (raw SIFT, or / 512) stay bit-exact (integer kernels)."""
    import torch

    from matching_sift_b200 import datagen

    q, r = datagen.make_workload(300, 4000, seed=11)
    d, i = oracle.brute_2nn_u8(q, r)
    for scale in (1.0, 1.0 / 512):
        out = ms.match(torch.from_numpy(q.astype(np.float32) * scale).to(cuda_device),
                       torch.from_numpy(r.astype(np.float32) * scale).to(cuda_device), outputs=("nn_idx", "nn_dist"))
        np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
        np.testing.assert_array_equal(out["nn_dist"].cpu().numpy().astype(np.float64),
                                      d.astype(np.float64) * scale * scale)


def _fp64_lsh(q, r, planes):
    """FP64 restatement of the LSH search on float rows: codes (bit j when the
    dot product with plane j is negative), the members of the query's bucket
    in each table, nearest by FP64 squared distance. Also flags, per point,
    whether any of its dot products is so close to 0 that FP32 and FP64 may
    disagree on the sign."""
    L, k = planes.shape[:2]
    q64, r64 = q.astype(np.float64), r.astype(np.float64)
    qc, rc, amb_q, amb_r = [], [], np.zeros(len(q), bool), np.zeros(len(r), bool)
    for t in range(L):
        p = planes[t].astype(np.float64)
        for x, codes, amb in ((q64, qc, amb_q), (r64, rc, amb_r)):
            d = x @ p.T
            bound = 1e-5 * (np.abs(x) @ np.abs(p).T)
            amb |= (np.abs(d) <= bound).any(1)
            codes.append(((d < 0).astype(np.int64) << np.arange(k)).sum(1))
    nn = np.full(len(q), -1, np.int64)
    nd = np.full(len(q), np.inf)
    for i in range(len(q)):
        member = np.zeros(len(r), bool)
        for t in range(L):
            member |= rc[t] == qc[t][i]
        idx = np.nonzero(member)[0]
        if len(idx):
            d = ((r64[idx] - q64[i]) ** 2).sum(1)
            j = np.lexsort((idx, d))[0]
            nn[i], nd[i] = idx[j], d[j]
    return nn, nd, amb_q, amb_r


def test_lsh_on_general_floats(cuda_device):
    """lsh_match / lsh_gpu on the reference benchmark's kind of data: the
    nearest bucket member equals the FP64 restatement's, except for queries
    whose buckets involve a point with a dot product at the FP32/FP64 sign
    boundary; distances within the float tolerance."""
    import torch

    from matching_sift_b200 import datagen

    q, r = rand_unit(400, 12), rand_unit(20000, 13)
    L, k = 2, 10
    planes = datagen.quantize_planes(datagen.make_hyperplanes(k, L, seed=14), 32.0)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    out = ms.lsh_match(qd, rd, torch.from_numpy(planes).to(cuda_device), threshold=0.0, candidates=True)
    assert ms.stream_status() == ms.SIFT_OK
    nn, nd, amb_q, amb_r = _fp64_lsh(q, r, planes)
    got = out["nn_idx"][:, 0].cpu().numpy().astype(np.int64)
    gd = out["nn_dist"][:, 0].cpu().numpy().astype(np.float64)
    clear = ~amb_q & ~amb_r[np.where(nn >= 0, nn, 0)] & ~amb_r[np.where(got >= 0, got, 0)]
    assert clear.mean() > 0.9
    np.testing.assert_array_equal(got[clear], nn[clear])
    ok = clear & (nn >= 0)
    qn = (q.astype(np.float64) ** 2).sum(1)
    assert (np.abs(gd[ok] - nd[ok]) <= TOL * 2 * qn[ok] + 1e-6).all()
    # the reference-named entry point with rand() +/-1 planes on float rows
    m = torch.zeros(400, dtype=torch.int32, device=cuda_device)
    assert ms.lsh_gpu(qd, rd, ms.FLOAT_DEVICE, 400, 20000, m, 0.8, None, 2, 3, 0, 12) == ms.SIFT_OK
    mm = m.cpu().numpy().view(np.uint32)
    assert ((mm < 20000) | (mm == 0xFFFFFFFF)).all() and (mm < 20000).mean() > 0.5


def test_lsh_on_general_floats_more_probes_never_lose_the_nearest(cuda_device):
    """Multi-probe LSH on general float rows: the probe codes of P probes are a
    prefix of those of more probes, so every added probe only adds candidates:
    the candidate count never falls and the nearest distance never grows, up to
    64 probes per table (more than a warp's 32 lanes)."""
    import torch

    from matching_sift_b200 import datagen

    q, r = rand_unit(300, 21), rand_unit(20000, 22)
    planes = torch.from_numpy(datagen.quantize_planes(datagen.make_hyperplanes(12, 2, seed=23), 32.0)).to(cuda_device)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    prev_d, prev_c = None, None
    for probes in (1, 8, 33, 64):
        o = ms.lsh_match(qd, rd, planes, threshold=0.0, probes=probes, candidates=True)
        assert ms.stream_status() == ms.SIFT_OK
        d1 = o["nn_dist"][:, 0].cpu().numpy().astype(np.float64)
        c = o["candidates"].cpu().numpy().astype(np.int64)
        if prev_d is not None:
            assert (c >= prev_c).all()
            assert (d1 <= prev_d).all()
        prev_d, prev_c = d1, c
    # every reported neighbour is a real row at its FP64 distance (within the float tolerance)
    idx = o["nn_idx"][:, 0].cpu().numpy().astype(np.int64)
    ok = idx >= 0
    dd = ((q[ok].astype(np.float64) - r[idx[ok]].astype(np.float64)) ** 2).sum(1)
    qn = (q.astype(np.float64) ** 2).sum(1)[ok]
    assert (np.abs(prev_d[ok] - dd) <= TOL * 2 * qn + 1e-6).all()
