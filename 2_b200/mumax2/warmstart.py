"""Learned warm start of batched relaxations.

  relax_pool   plain relax() of many problems through one batched plan with continuous
               batching (a finished slot takes the next problem at once)
  generate     relaxed states of seeded problems, kept on the GPU as training data
  train        the U-Net (unet.py) on them with this library's kernels
  predict      initial states for new problems, batched
  evaluate     cold vs warm relaxations of held-out problems: rate, steps, and the
               final state judged against the cold relax (max torque and energy); a warm
               start that fails falls back to the cold start
"""
import time

import numpy as np

from . import unet as U
from . import workloads as W


def relax_pool(problem, sims, masks, states, thr, slots=256, maxerr=1e-6, max_steps=100000, device=0,
               keep_states=False, plan=None):
    """Relaxes problem q from states[q] until maxtorque < thr[q].  Returns a dict of
    arrays: steps, maxtorque, energy (J) and, with keep_states, the relaxed states."""
    import torch
    from .plan import Plan
    n = problem["n"]
    N = int(np.prod(n))
    nq = len(sims)
    B = min(slots, nq)
    own = plan is None
    if own:
        plan = Plan(problem, masks={"msat": np.concatenate(masks[:B])}, sims=sims[:B], masks_per_sim=True,
                    device=device)
    plan.solver("rk23", dt=1e-14, maxerr=maxerr)
    mt = plan.mask_tensor("msat")
    slot = [-1] * B
    nxt = 0
    res = {"steps": np.zeros(nq, dtype=np.int64), "maxtorque": np.zeros(nq), "energy": np.zeros(nq)}
    if keep_states:
        res["state"] = np.zeros((nq, 3 * N), dtype=np.float32)

    def fill(free):
        nonlocal nxt
        idx, jobs = [], []
        for b in free:
            if nxt >= nq:
                break
            mt[b * N:(b + 1) * N].copy_(torch.from_numpy(np.asarray(masks[nxt], dtype=np.float32)))
            slot[b] = nxt
            idx.append(b)
            jobs.append(nxt)
            nxt += 1
        if idx:
            plan.batch_restart(idx, np.stack([states[q] for q in jobs]), np.asarray(thr)[jobs],
                               sims=[sims[q] for q in jobs], max_steps=max_steps)

    fill(range(B))
    done = 0
    refill = max(1, B // 8)
    while done < nq:
        plan.batch_drive(target_active=max(0, B - refill) if nxt < nq else 0,
                         max_attempts=0)
        st = plan.batch_stats()
        free = [b for b in range(B) if slot[b] >= 0 and st[b]["done"]]
        if not free:
            continue
        en = plan.batch_energy()
        state = plan.get_state() if keep_states else None
        for b in free:
            q = slot[b]
            res["steps"][q] = st[b]["step"]
            res["maxtorque"][q] = st[b]["maxtorque"]
            res["energy"][q] = en[b][4]
            if keep_states:
                res["state"][q] = state[3 * N * b:3 * N * (b + 1)]
            slot[b] = -1
            done += 1
        fill(free)
    if own:
        plan.close()
    return res


def thresholds(sims, gamma=2.211e5, rel=1e-4):
    return np.array([rel * gamma * s["msat"] for s in sims])


class Dataset:
    """Features, targets and masks of relaxed problems, resident on the GPU."""

    def __init__(self, problem, sims, masks, states, device=0):
        import torch
        n = problem["n"]
        self.n = n
        self.P = n[1] * n[2]
        dev = torch.device("cuda", device)
        self.feats = torch.tensor(U.features(sims, masks, n), device=dev)
        self.targets = torch.tensor(np.stack([U.target_from_state(s, n) for s in states]), device=dev)
        self.masks = torch.tensor(np.stack([np.asarray(m, dtype=np.float32) for m in masks]), device=dev)

    def __len__(self):
        return self.feats.shape[0]


def generate(nsim, seed, slots=256, device=0):
    """Seeded relaxation problems relaxed from the cold start: (problem, sims, masks, result)."""
    problem, sims, masks = W.relax_set(nsim, seed=seed)
    cold = W.cold_state(problem["n"], 1)
    res = relax_pool(problem, sims, masks, [cold] * nsim, thresholds(sims), slots=slots, device=device,
                     keep_states=True)
    return problem, sims, masks, res


def train(data, epochs=20, batch=256, lr=1e-3, seed=0, device=0, log=None):
    """Adam with a short linear warm-up and a cosine decay; returns (net, losses per epoch)."""
    import torch
    H, Wd = data.n[1], data.n[2]
    net = U.UNet(batch, H, Wd, device=device, seed=seed)
    rng = np.random.default_rng(seed)
    nb = len(data) // batch
    losses = []
    total = epochs * nb
    k = 0
    for ep in range(epochs):
        perm = torch.tensor(rng.permutation(len(data))[:nb * batch], device=data.feats.device)
        acc = torch.zeros((), device=data.feats.device)
        for i in range(nb):
            idx = perm[i * batch:(i + 1) * batch]
            net.set_input(data.feats[idx])
            net.forward()
            net.set_target(data.targets[idx], data.masks[idx])
            acc += net.loss_and_grad()[0]
            net.backward()
            warm = min(1.0, (k + 1) / max(1, total // 20))
            net.adam(lr=lr * warm * 0.5 * (1 + np.cos(np.pi * k / total)))
            k += 1
        losses.append(float(acc.item()) / nb)
        if log:
            log(ep, losses[-1])
    return net, losses


def predict(net, sims, masks, n):
    """Initial states (internal SoA, normalised, masked) for the problems, net.B per launch;
    the features are built once and kept on the GPU."""
    import torch
    B = net.B
    feats = torch.tensor(U.features(sims, masks, n), device=net.device)
    if len(sims) % B:
        pad = torch.zeros((B - len(sims) % B,) + tuple(feats.shape[1:]), device=net.device)
        feats = torch.cat([feats, pad])
    out = []
    for i in range(0, len(sims), B):
        net.set_input(feats[i:i + B])
        net.forward()
        o = net.output3()[:min(B, len(sims) - i)]
        out.append(U.state_from_output(o, np.stack(masks[i:i + B])))
    return np.concatenate(out)


def choose_starts(problem, sims, masks, candidates, slots=256, device=0, plan=None):
    """Per problem, the candidate start of lowest energy (the judge of a predicted start:
    a prediction above the cold start's energy is not used).  candidates: list of
    [nq][3N] arrays; returns (states, index of the chosen candidate per problem)."""
    from .plan import Plan
    import torch
    n = problem["n"]
    N = int(np.prod(n))
    nq = len(sims)
    B = min(slots, nq)
    own = plan is None
    if own:
        plan = Plan(problem, masks={"msat": np.concatenate(masks[:B])}, sims=sims[:B], masks_per_sim=True,
                    device=device)
    mt = plan.mask_tensor("msat")
    energies = np.zeros((len(candidates), nq))
    for i in range(0, nq, B):
        k = min(B, nq - i)
        mt[:k * N].copy_(torch.from_numpy(np.concatenate(masks[i:i + k])))
        plan.set_sims(sims[i:i + k] + sims[i:i + 1] * (plan.nsim - k))
        for c, cand in enumerate(candidates):
            st = np.zeros((plan.nsim, 3 * N), dtype=np.float32)
            st[:k] = cand[i:i + k]
            plan.set_state(st.ravel())
            energies[c, i:i + k] = plan.batch_energy()[:k, 4]
    if own:
        plan.close()
    pick = np.argmin(energies, axis=0)
    states = np.stack([candidates[pick[q]][q] for q in range(nq)])
    return states, pick


def evaluate(net, problem, sims, masks, slots=256, device=0, energy_tol=1e-4, max_steps=20000):
    """Cold and warm relaxations of the same problems (times include the network's
    inference for the warm start).  A warm relax that does not reach the threshold within
    max_steps, or ends above the cold relax's energy by more than energy_tol (relative),
    counts as failed and is redone from the cold start (time included)."""
    import torch
    from .plan import Plan
    n = problem["n"]
    thr = thresholds(sims)
    cold = W.cold_state(n, 1)
    B = min(slots, len(sims))
    plan = Plan(problem, masks={"msat": np.concatenate(masks[:B])}, sims=sims[:B], masks_per_sim=True,
                device=device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = relax_pool(problem, sims, masks, [cold] * len(sims), thr, slots=slots, device=device, plan=plan)
    torch.cuda.synchronize()
    t_cold = time.perf_counter() - t0
    t0 = time.perf_counter()
    pred = predict(net, sims, masks, n)
    init, pick = choose_starts(problem, sims, masks, [pred, np.repeat(cold[None, :], len(sims), axis=0)],
                               slots=slots, device=device, plan=plan)
    torch.cuda.synchronize()
    t_inf = time.perf_counter() - t0
    rw = relax_pool(problem, sims, masks, list(init), thr, slots=slots, device=device, max_steps=max_steps,
                    plan=plan)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0
    conv = rw["maxtorque"] < thr
    erel = np.abs(rw["energy"] - rc["energy"]) / np.maximum(np.abs(rc["energy"]), 1e-30)
    ok = conv & ((rw["energy"] <= rc["energy"]) | (erel <= energy_tol))
    fail = np.nonzero(~ok)[0]
    t_fb = 0.0
    if len(fail):
        t1 = time.perf_counter()
        relax_pool(problem, [sims[q] for q in fail], [masks[q] for q in fail], [cold] * len(fail), thr[fail],
                   slots=slots, device=device, plan=plan)
        torch.cuda.synchronize()
        t_fb = time.perf_counter() - t1
    plan.close()
    return {
        "relaxations": len(sims),
        "cold_per_s": len(sims) / t_cold, "warm_per_s": len(sims) / (t_warm + t_fb),
        "speedup": t_cold / (t_warm + t_fb),
        "cold_steps_mean": float(rc["steps"].mean()), "warm_steps_mean": float(rw["steps"].mean()),
        "steps_saved_frac": float(1 - rw["steps"].sum() / max(1, rc["steps"].sum())),
        "inference_s": t_inf, "predicted_start_used_frac": float((pick == 0).mean()),
        "warm_ok_frac": float(ok.mean()), "fallbacks": int(len(fail)),
        "energy_within_tol_frac": float((erel <= energy_tol).mean()),
        "energy_rel_median": float(np.median(erel)),
        "warm_lower_energy_frac": float((rw["energy"] < rc["energy"]).mean()),
    }
