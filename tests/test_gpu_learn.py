"""Learned initial guess: the tensor-core convolutions against a plain
PyTorch FP32 reference of the same net, the parameter gradient against
torch autograd, and the online record/train/use loop inside time steps
against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from bluebottle_b200 import Sim, configs
from oracle.orc import Oracle
from tests.helpers import rel_err, field_interior

pytestmark = pytest.mark.gpu

NL, NT, NC = 4, 27, 16


def _torch():
    import torch
    return torch


def _params(seed, scale=0.35):
    """Random parameters in the library's layout: W[l][t][cout][cin] then
    b[l][cout]; padded input channels of layer 1 and outputs 1..15 of
    layer 4 stay zero, as the library keeps them."""
    rng = np.random.default_rng(seed)
    W = np.zeros((NL, NT, NC, NC), np.float32)
    b = np.zeros((NL, NC), np.float32)
    for l in range(NL):
        cin = 4 if l == 0 else NC
        cout = 1 if l == NL - 1 else NC
        W[l, :, :cout, :cin] = rng.standard_normal((NT, cout, cin)) * scale / np.sqrt(27 * cin / 4)
        b[l, :cout] = 0.1 * rng.standard_normal(cout)
    return W, b


def _set_params(lib, W, b):
    flat = np.concatenate([W.ravel(), b.ravel()]).astype(np.float32)
    assert lib.bbb_learn_param_count() == flat.size
    rc = lib.bbb_learn_set_params(flat.ctypes.data_as(C.POINTER(C.c_float)), flat.size)
    assert rc == 0


def _bf16(t):
    return t.to(_torch().bfloat16).to(_torch().float32)


def _torch_net(feat, W, b, dims, periodic, emulate_bf16=True):
    """feat: (n, 16) float32, cells x fastest; returns (n,) output."""
    torch = _torch()
    import torch.nn.functional as F
    nx, ny, nz = dims
    x = feat.reshape(nz, ny, nx, NC).permute(3, 0, 1, 2).unsqueeze(0)
    for l in range(NL):
        w = torch.from_numpy(W[l]).reshape(3, 3, 3, NC, NC)   # [dz][dy][dx][o][c]
        w = w.permute(3, 4, 0, 1, 2).contiguous()             # [o][c][dz][dy][dx]
        if emulate_bf16:
            w = _bf16(w)
        xp = x
        # pad x, y, z (last three dims are z, y, x)
        for dim, per in ((4, periodic[0]), (3, periodic[1]), (2, periodic[2])):
            if per:
                lo = xp.narrow(dim, xp.shape[dim] - 1, 1)
                hi = xp.narrow(dim, 0, 1)
            else:
                lo = torch.zeros_like(xp.narrow(dim, 0, 1))
                hi = lo
            xp = torch.cat([lo, xp, hi], dim=dim)
        z = F.conv3d(xp, w) + torch.from_numpy(b[l]).reshape(1, NC, 1, 1, 1)
        if l < NL - 1:
            x = F.gelu(z, approximate="tanh")
            if emulate_bf16:
                x = _bf16(x)
        else:
            x = z
    return x[0, 0].reshape(-1)


def _prepared_sim():
    sim = Sim(configs.taylor_green(32))
    try:
        sim.prepare()
        assert sim.lib.bbb_learn_enable(0) == 0
    except BaseException:
        sim.close()
        raise
    return sim


def _features(n, seed):
    torch = _torch()
    g = torch.Generator().manual_seed(seed)
    f = torch.zeros(n, NC)
    f[:, :3] = torch.rand(n, 3, generator=g) * 2 - 1
    f[:, 3] = (torch.rand(n, generator=g) < 0.1).float()
    return _bf16(f)


@pytest.mark.parametrize("dims,periodic", [((256, 6, 5), (1, 1, 1)),
                                           ((200, 4, 3), (0, 0, 0)),
                                           ((64, 5, 4), (1, 0, 1))])
def test_forward_tensor_cores_match_torch(gpu, dims, periodic):
    torch = _torch()
    sim = _prepared_sim()
    try:
        lib = sim.lib
        W, b = _params(1)
        _set_params(lib, W, b)
        n = dims[0] * dims[1] * dims[2]
        feat = _features(n, 2)
        fd = feat.to(torch.bfloat16).cuda().contiguous()
        outs = {}
        for ref in (0, 1):
            od = torch.zeros(n, dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            rc = lib.bbb_learn_forward(*dims, *periodic, C.c_void_p(fd.data_ptr()),
                                       C.c_void_p(od.data_ptr()), ref)
            assert rc == 0
            outs[ref] = od.cpu()
        expect = _torch_net(feat, W, b, dims, periodic)
        scale = expect.abs().max().item()
        assert scale > 0.05
        e_tc = (outs[0] - expect).abs().max().item() / scale
        e_ref = (outs[1] - expect).abs().max().item() / scale
        assert e_ref < 2e-2, e_ref
        assert e_tc < 2e-2, e_tc
        assert (outs[0] - outs[1]).abs().max().item() / scale < 2e-2
    finally:
        sim.close()


def test_parameter_gradient_matches_autograd(gpu):
    torch = _torch()
    sim = _prepared_sim()
    try:
        lib = sim.lib
        W, b = _params(3, scale=0.3)
        _set_params(lib, W, b)
        cx, cy, cz, nb, margin = 128, 10, 10, 2, 4
        n = cx * cy * cz * nb
        feat = _features(n, 4)
        g = torch.Generator().manual_seed(5)
        tgt = torch.randn(n, generator=g) * 0.2
        fd = feat.to(torch.bfloat16).cuda().contiguous()
        td = tgt.cuda().contiguous()
        grad = np.zeros(lib.bbb_learn_param_count(), np.float32)
        torch.cuda.synchronize()
        loss = lib.bbb_learn_grad(cx, cy, cz, nb, margin, C.c_void_p(fd.data_ptr()),
                                  C.c_void_p(td.data_ptr()),
                                  grad.ctypes.data_as(C.POINTER(C.c_float)))
        assert loss > 0
        # torch autograd in FP32 on the same stacked box (zero padding)
        Wt = torch.tensor(W, requires_grad=True)
        bt = torch.tensor(b, requires_grad=True)
        import torch.nn.functional as F
        x = feat.reshape(cz * nb, cy, cx, NC).permute(3, 0, 1, 2).unsqueeze(0)
        for l in range(NL):
            w = Wt[l].reshape(3, 3, 3, NC, NC).permute(3, 4, 0, 1, 2)
            z = F.conv3d(x, w, padding=1) + bt[l].reshape(1, NC, 1, 1, 1)
            x = F.gelu(z, approximate="tanh") if l < NL - 1 else z
        out = x[0, 0]
        m = torch.zeros(cz * nb, cy, cx, dtype=torch.bool)
        for q in range(nb):
            m[q * cz + margin:(q + 1) * cz - margin, margin:cy - margin,
              margin:cx - margin] = True
        d = out[m] - tgt.reshape(cz * nb, cy, cx)[m]
        L = (d * d).mean()
        L.backward()
        gref = np.concatenate([Wt.grad.numpy().ravel(), bt.grad.numpy().ravel()])
        assert abs(loss - L.item()) / L.item() < 2e-2
        cos = float(np.dot(grad, gref) / (np.linalg.norm(grad) * np.linalg.norm(gref)))
        rel = float(np.linalg.norm(grad - gref) / np.linalg.norm(gref))
        assert cos > 0.999 and rel < 5e-2, (cos, rel)
        # per layer, too
        for l in range(NL):
            a = grad[l * NT * NC * NC:(l + 1) * NT * NC * NC]
            r = gref[l * NT * NC * NC:(l + 1) * NT * NC * NC]
            assert np.linalg.norm(a - r) <= 6e-2 * np.linalg.norm(r) + 1e-9, l
    finally:
        sim.close()


def test_online_record_train_use_keeps_parity(gpu):
    """Sedimentation 128x32x32, 4 spheres: record crops for 3 steps, train,
    then step with the gated guess on; the fields still match the FP64
    oracle (which starts every solve from phi_prev) to solver tolerance."""
    wl = configs.sedimentation((128, 32, 32), (32.0, 8.0, 8.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=4)
    sim = Sim(wl, options=dict(lamb_max_iter_override=2, learned_guess=1))
    try:
        orc = Oracle.from_sim(sim)
    except BaseException:
        sim.close()
        raise
    try:
        sim.prepare()
        lib = sim.lib
        for _ in range(3):
            sim.step()
            orc.step()
        assert lib.bbb_learn_crops() >= 16
        l0 = lib.bbb_learn_train(1, 1e-3)
        l1 = lib.bbb_learn_train(60, 1e-3)
        assert 0 <= l1 < l0, (l0, l1)
        assert lib.bbb_learn_enable(3) == 0
        used = 0
        for _ in range(2):
            sim.step()
            orc.step()
            st = sim.stats()
            used += st.guess_used
            assert st.extrap_r0 > 0
            if st.guess_used:
                assert st.guess_r0 < st.extrap_r0
        sim.pull()
        d = sim.dom
        for nm in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, nm, sim.array(nm)),
                        field_interior(d, nm, orc.field(nm)))
            assert e < 1e-7, (nm, e)
        assert sim.status() == 0
    finally:
        sim.close()
        orc.close()


def test_cost_gate_times_and_skips(gpu):
    """Mode bit 4: the evaluated step reports the guess's device cost and
    the estimated saving of the solve after it; when the saving does not
    exceed the cost the next steps skip the evaluation (the solve starts
    from phi_prev, as the reference's does), otherwise they evaluate."""
    wl = configs.sedimentation((128, 32, 32), (32.0, 8.0, 8.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=4)
    sim = Sim(wl, options=dict(lamb_max_iter_override=2, learned_guess=1))
    try:
        sim.prepare()
        lib = sim.lib
        for _ in range(3):
            sim.step()
        lib.bbb_learn_train(30, 1e-3)
        assert lib.bbb_learn_enable(2 | 4) == 0
        sim.step()
        st = sim.stats()
        assert st.guess_evaluated == 1 and st.guess_cost_ms > 0
        assert st.guess_benefit_ms >= 0
        if st.guess_used == 0:
            assert st.guess_benefit_ms == 0
        pays = st.guess_benefit_ms > st.guess_cost_ms
        for _ in range(2):
            sim.step()
            st = sim.stats()
            assert st.guess_evaluated == (1 if pays else 0)
            if not pays:
                assert st.guess_used == 0
            pays = pays and st.guess_benefit_ms > st.guess_cost_ms
        assert sim.status() == 0
    finally:
        sim.close()


def test_trained_guess_saves_iterations_on_a_held_out_step(gpu, tmp_path):
    """What the trained net gains over the method without it, on a step it
    was not trained on.  A 64^3 sedimentation case (16 spheres, FP32 inner
    solves, tolerance 1e-8) records crops for 16 steps and trains on them
    online; the state after those steps goes to the reference's restart
    file.  The next step then runs twice from that state: once with its
    first Poisson solve started from the learned guess, once (a fresh
    simulation read back from the restart file) from the extrapolation
    phi_prev, where the reference starts it.  The guess starts at a lower
    FP64 residual and its solve needs fewer BiCGSTAB iterations to the same
    tolerance; the two steps' fields agree to what the tolerance allows."""
    path = str(tmp_path / "restart.config")
    wl = configs.sedimentation((64, 64, 64), (16.0, 16.0, 16.0), 16, nu=0.05,
                               lamb_max_iter=1, seed=11, prec=1,
                               gap=configs.DENSE_GAP, loa=configs.DENSE_LOA)
    opts = dict(lamb_max_iter_override=1, learned_guess=1)
    names = ("u", "v", "w", "p")
    sim = Sim(wl, options=opts)
    try:
        sim.prepare()
        lib = sim.lib
        assert lib.bbb_learn_enable(1) == 0
        for k in range(16):
            sim.step()
            if k % 4 == 3:
                lib.bbb_learn_train(60, 1e-3)
        assert lib.bbb_learn_train(400, 1e-3) >= 0
        sim.pull()
        sim.out_restart(path)
        assert lib.bbb_learn_enable(2) == 0
        sim.step()
        st = sim.stats()
        assert st.guess_evaluated == 1
        guess = dict(used=st.guess_used, r0=st.guess_r0, ext=st.extrap_r0,
                     iters=st.pp_iters_first)
        sim.pull()
        d = sim.dom
        fg = {nm: field_interior(d, nm, sim.array(nm)).copy() for nm in names}
    finally:
        sim.close()
    sim = Sim(wl, options=opts)
    try:
        sim.prepare()
        sim.in_restart(path)
        sim.push()
        assert sim.lib.bbb_learn_enable(0) == 0
        sim.step()
        plain_iters = sim.stats().pp_iters_first
        sim.pull()
        d = sim.dom
        fp = {nm: field_interior(d, nm, sim.array(nm)).copy() for nm in names}
    finally:
        sim.close()
    print("held-out step: guess r0 %.3e vs extrapolation %.3e, first solve "
          "%d vs %d iterations" % (guess["r0"], guess["ext"], guess["iters"],
                                   plain_iters))
    assert guess["used"] == 1 and guess["r0"] < guess["ext"]
    assert 0 < guess["iters"] < plain_iters, (guess, plain_iters)
    for nm in names:
        assert rel_err(fg[nm], fp[nm]) < 1e-6, nm
