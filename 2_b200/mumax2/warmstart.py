"""Learned warm start of batched relaxations of 64x64x1 films.

  relax_pool   plain relax() of many problems through one batched plan with continuous
               batching (a finished slot takes the next problem at once)
  generate     relaxed states of seeded problems, kept on the GPU as training data
  train        the U-Net (unet.py) on them with this library's kernels
  predict      initial states for new problems, batched, built and kept on the GPU
  evaluate     cold vs warm relaxations of held-out problems: rate, steps, and the
               final state checked against the cold relax (max torque and energy); a warm
               start that fails is redone from the cold start in the same pool
"""
import time

import numpy as np

from . import _native as nat
from . import unet as U
from . import workloads as W


def _tail_plan(plan, problem, masks0, sims0, slots, device, maxerr):
    """The small plan (same geometry, `slots` simulations) that finishes a pool's last
    relaxations; made once per main plan."""
    from .plan import Plan
    t = getattr(plan, "_tail_plan", None)
    if t is None or t.nsim != slots:
        t = Plan(problem, masks={"msat": np.concatenate([masks0] * slots)}, sims=[sims0] * slots,
                 masks_per_sim=True, device=device)
        plan._tail_plan = t
    t.solver("rk23", dt=1e-14, maxerr=maxerr)
    return t


def relax_pool(problem, sims, masks, states, thr, slots=256, maxerr=1e-6, max_steps=100000, device=0,
               keep_states=False, plan=None, accept=None, fallback=None, fallback_max_steps=100000,
               tail_slots=16, want_energy=True, spec_steps=0, order=None, masks_dev=None):
    """Relaxes problem q from states[q] until maxtorque < thr[q].  states: a list of host
    arrays or a float32 device tensor [nq][3N].  Returns a dict of arrays: steps,
    maxtorque, energy (J; zeros without want_energy, which accept needs) and, with
    keep_states, the relaxed states.

    accept(q, steps, maxtorque, energy) -> bool and fallback (one host state): a relax that
    accept rejects is redone, in the same pool, from the fallback state with
    fallback_max_steps as its step limit; the result arrays then hold the fallback's
    result, "first_*" arrays the first attempt's and "fell_back" marks the problems
    concerned.  Without spec_steps the redo is queued when the first attempt is rejected.
    With spec_steps > 0 the redo of a problem starts speculatively, in a free slot beside
    the first attempt, once that attempt has run spec_steps steps: the long first attempts
    are the ones the step limit rejects, and their redo then no longer waits for them.  An
    accepted first attempt cancels its redo; a rejected one takes the redo's result,
    whenever it ends.  Each run is the same computation either way, so the results do not
    depend on spec_steps ("spec_started" / "spec_cancelled" count the speculative runs).

    Drain phase: once nothing is queued and at most tail_slots relaxations are left, they
    move (state, scalars, mask and steps so far) to a plan of tail_slots simulations,
    whose launches carry that many simulations' blocks instead of the pool's (a step of
    the 256-slot pool costs about the same with one slot active as with all).  The moved
    relaxations restart their step-size control from dt = 1e-14 s.

    order (optional): the problems in the order the pool starts them (default 0..nq-1);
    starting the longest relaxations first keeps them from forming the pool's end.
    masks_dev (optional): the problems' masks already on the device ([nq][N] float32)."""
    import collections
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
    on_dev = hasattr(states, "data_ptr")
    speculate = bool(spec_steps) and accept is not None and fallback is not None
    queue = collections.deque((int(q), False) for q in (range(nq) if order is None else order))
    res = {"steps": np.zeros(nq, dtype=np.int64), "maxtorque": np.zeros(nq), "energy": np.zeros(nq)}
    if accept is not None:
        res.update({"first_steps": np.zeros(nq, dtype=np.int64), "first_maxtorque": np.zeros(nq),
                    "first_energy": np.zeros(nq), "fell_back": np.zeros(nq, dtype=bool)})
    if keep_states:
        res["state"] = np.zeros((nq, 3 * N), dtype=np.float32)
    thr = np.asarray(thr)
    # per slot of the current plan: problem, redo flag, steps done before this plan
    cur = plan
    nslot = B
    slot, retry, offset = [-1] * nslot, [False] * nslot, [0] * nslot
    spec_slot = {}      # problem -> slot of its speculative redo while the first attempt runs
    spec_result = {}    # problem -> result of a speculative redo that ended first
    awaiting = set()    # problems whose first attempt was rejected while their redo runs
    n_spec, n_cancel = 0, 0

    dev = plan.mask_tensor("msat").device

    def to_dev(a):
        """One host-to-device copy of a stack of host arrays (states or masks)."""
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)

    def pick_masks(qs):
        """The masks of problems qs on the device: gathered from masks_dev when the caller
        keeps them there, else uploaded in one copy."""
        if masks_dev is not None:
            return masks_dev[torch.tensor(qs, device=masks_dev.device)]
        return to_dev(np.stack([np.asarray(masks[q], dtype=np.float32) for q in qs]))

    def restart(idx, m0, jobs, limits):
        if not hasattr(m0, "data_ptr"):
            m0 = to_dev(m0)
        cur.batch_restart(idx, m0, thr[jobs], sims=[sims[q] for q in jobs], max_steps=limits)

    def place(bs, qs, is_fb):
        """Slots bs take problems qs: their masks in one copy, and the slot records."""
        mt = cur.mask_tensor("msat").view(-1, N)
        mt[torch.tensor(bs, device=dev)] = pick_masks(qs)
        for b, q, f in zip(bs, qs, is_fb):
            slot[b], retry[b], offset[b] = q, f, 0

    def fill(free):
        idx, jobs, fb = [], [], []
        for b in free:
            if not queue:
                break
            q, is_fb = queue.popleft()
            idx.append(b)
            jobs.append(q)
            fb.append(is_fb)
        if not idx:
            return
        place(idx, jobs, fb)
        for flag, limit in ((False, max_steps), (True, fallback_max_steps)):
            sel = [k for k in range(len(idx)) if fb[k] == flag]
            if not sel:
                continue
            js = [jobs[k] for k in sel]
            if flag:
                m0 = np.stack([fallback] * len(js))
            elif on_dev:
                m0 = states[torch.tensor(js, device=states.device)]
            else:
                m0 = np.stack([states[q] for q in js])
            restart([idx[k] for k in sel], m0, js, limit)

    def migrate(st):
        """Moves the running relaxations of the pool into the tail plan."""
        nonlocal cur, nslot, slot, retry, offset
        run = [b for b in range(nslot) if slot[b] >= 0]
        state = cur.get_state()
        tail = _tail_plan(plan, problem, masks[0], sims[0], tail_slots, device, maxerr)
        mt = tail.mask_tensor("msat").view(-1, N)
        if run:
            mt[:len(run)] = pick_masks([slot[b] for b in run])
        new_slot, new_retry, new_off = [-1] * tail_slots, [False] * tail_slots, [0] * tail_slots
        m0, js, limits = [], [], []
        for i, b in enumerate(run):
            q = slot[b]
            new_slot[i], new_retry[i] = q, retry[b]
            new_off[i] = offset[b] + st[b]["step"]
            if retry[b] and spec_slot.get(q) == b:
                spec_slot[q] = i
            m0.append(state[3 * N * b:3 * N * (b + 1)])
            js.append(q)
            limits.append(max(1, (fallback_max_steps if retry[b] else max_steps) - new_off[i]))
        cur.batch_cancel(run)
        cur, nslot = tail, tail_slots
        slot, retry, offset = new_slot, new_retry, new_off
        # one restart per distinct remaining step limit
        for lim in sorted(set(limits)):
            sel = [i for i in range(len(run)) if limits[i] == lim]
            restart(sel, np.stack([m0[i] for i in sel]), [js[i] for i in sel], lim)

    def record(q, r, first=False):
        pre = "first_" if first else ""
        res[pre + "steps"][q], res[pre + "maxtorque"][q], res[pre + "energy"][q] = r[0], r[1], r[2]
        if not first and keep_states:
            res["state"][q] = r[3]

    fill(range(B))
    done = 0
    refill = max(1, B // 8)
    t_drive = 0.0
    t_all = time.perf_counter()
    while done < nq:
        t1 = time.perf_counter()
        # with speculation the host looks at the running attempts' steps every 64 attempts
        # (a drive that stops at that cap reports MM_ERR_TIMEOUT)
        cap = 64 if speculate else 0
        if cur is plan:
            drain = tail_slots if nslot > tail_slots else 0
            target = max(0, nslot - refill) if queue else drain
        else:
            target = max(0, nslot - 1) if queue else 0
        try:
            cur.batch_drive(target_active=target, max_attempts=cap)
        except nat.MMError as e:
            if not (cap and e.code == nat.MM_ERR_TIMEOUT):
                raise
        t_drive += time.perf_counter() - t1
        st = cur.batch_stats()
        ended = [b for b in range(nslot) if slot[b] >= 0 and st[b]["done"]]
        ended.sort(key=lambda b: retry[b])          # first attempts before redos
        free = []
        if ended:
            en = cur.batch_energy() if (want_energy or accept is not None) else None
            state = cur.get_state() if keep_states else None
            for b in ended:
                if slot[b] < 0:                     # a redo cancelled by its first attempt above
                    continue
                q = slot[b]
                r = (offset[b] + st[b]["step"], st[b]["maxtorque"], en[b][4] if en is not None else 0.0,
                     state[3 * N * b:3 * N * (b + 1)] if keep_states else None)
                slot[b] = -1
                free.append(b)
                if not retry[b]:
                    record(q, r)
                    if accept is None:
                        done += 1
                        continue
                    record(q, r, first=True)
                    if accept(q, r[0], r[1], r[2]):
                        done += 1
                        s = spec_slot.pop(q, None)
                        if s is not None:           # its redo is not needed
                            cur.batch_cancel([s])
                            slot[s] = -1
                            free.append(s)
                            n_cancel += 1
                        spec_result.pop(q, None)
                        continue
                    res["fell_back"][q] = True
                    if q in spec_result:
                        record(q, spec_result.pop(q))
                        done += 1
                    elif q in spec_slot:
                        awaiting.add(q)
                    else:
                        queue.appendleft((q, True))
                else:
                    if q in awaiting:
                        awaiting.discard(q)
                        spec_slot.pop(q, None)
                        record(q, r)
                        done += 1
                    elif spec_slot.get(q) == b:     # the redo ended before the first attempt
                        spec_slot.pop(q)
                        spec_result[q] = r
                    else:
                        record(q, r)
                        done += 1
        if speculate:
            idle = sorted(set(free) | {b for b in range(nslot) if slot[b] < 0 and st[b]["done"]})
            long_first = sorted((b for b in range(nslot) if slot[b] >= 0 and not retry[b]
                                 and slot[b] not in spec_slot and slot[b] not in spec_result
                                 and offset[b] + st[b]["step"] >= spec_steps), key=lambda b: -st[b]["step"])
            started = []
            for b in long_first:
                if not idle:
                    break
                started.append((idle.pop(0), slot[b]))
            if started:
                place([f for f, _ in started], [q for _, q in started], [True] * len(started))
                for f, q in started:
                    spec_slot[q] = f
                restart([f for f, _ in started], np.stack([fallback] * len(started)), [q for _, q in started],
                        fallback_max_steps)
                n_spec += len(started)
                free = [b for b in free if slot[b] < 0]
        fill(free)
        running = sum(1 for b in range(nslot) if slot[b] >= 0)
        if cur is plan and nslot > tail_slots and not queue and 0 < running <= tail_slots:
            migrate(cur.batch_stats())
    res["drive_s"] = t_drive
    res["host_s"] = time.perf_counter() - t_all - t_drive
    res["spec_started"], res["spec_cancelled"] = n_spec, n_cancel
    if own:
        t = getattr(plan, "_tail_plan", None)
        if t is not None:
            t.close()
        plan.close()
    return res


def step_budget(train_steps, q=99.0):
    """Step budget of a warm relax: the q-th percentile of the cold relaxations' step counts
    over the training problems (a warm start that needs more is stuck in a slow mode and
    falls back to the cold start)."""
    return int(np.ceil(np.percentile(np.asarray(train_steps), q)))


def thresholds(sims, gamma=2.211e5, rel=1e-4):
    return np.array([rel * gamma * s["msat"] for s in sims])


class Dataset:
    """Features, targets and masks of relaxed problems, resident on the GPU.

    mirror=True adds, for every relaxed problem, its mirror image x -> -x: mask and
    fields reflected along x, the in-plane field and anisotropy axis (Bx, By) -> (Bx, -By),
    (ux, uy) -> (ux, -uy), and the relaxed state m -> (mx, -my, -mz) at the mirrored cell.
    Magnetisation and field are axial vectors, so a mirror R acts on them as -det(R) R =
    diag(1, -1, -1) here; the LLG equation, every energy term, the grid and the cold start
    (uniform +x) are invariant under this map, so the mirrored state is exactly what the
    plain relaxer gives for the mirrored problem.  (The other flips and rotations of the
    square map the +x cold start to another direction and are not used: where a problem
    has several minima, the relaxer's choice depends on the start.)"""

    def __init__(self, problem, sims, masks, states, device=0, mirror=False):
        import torch
        n = problem["n"]
        self.n = n
        self.P = n[1] * n[2]
        dev = torch.device("cuda", device)
        self.feats = torch.tensor(U.features(sims, masks, n), device=dev)
        self.targets = torch.tensor(np.stack([U.target_from_state(s, n) for s in states]), device=dev)
        mk = np.stack([np.asarray(m, dtype=np.float32) for m in masks])
        self.masks = torch.tensor(mk, device=dev)
        self.mask_counts = mk.sum(axis=1).astype(np.float64)   # host copy: no device read per batch
        if mirror:
            ny, nx = n[1], n[2]
            f = torch.flip(self.feats.view(-1, ny, nx, self.feats.shape[-1]), dims=[2]).reshape(self.feats.shape)
            f = f.clone()
            f[:, :, U.FEAT_AXIS_Y] *= -1.0   # (ux, uy) -> (ux, -uy)
            f[:, :, U.FEAT_B_Y] *= -1.0      # (Bx, By) -> (Bx, -By)
            t = torch.flip(self.targets.view(-1, ny, nx, 3), dims=[2]).reshape(self.targets.shape).clone()
            t[:, :, 1] *= -1.0
            t[:, :, 2] *= -1.0
            m2 = torch.flip(self.masks.view(-1, ny, nx), dims=[2]).reshape(self.masks.shape)
            self.feats = torch.cat([self.feats, f])
            self.targets = torch.cat([self.targets, t])
            self.masks = torch.cat([self.masks, m2])
            self.mask_counts = np.concatenate([self.mask_counts, self.mask_counts])

    def __len__(self):
        return self.feats.shape[0]


def generate(nsim, seed, slots=256, device=0):
    """Seeded relaxation problems relaxed from the cold start: (problem, sims, masks, result)."""
    problem, sims, masks = W.relax_set(nsim, seed=seed)
    cold = W.cold_state(problem["n"], 1)
    res = relax_pool(problem, sims, masks, [cold] * nsim, thresholds(sims), slots=slots, device=device,
                     keep_states=True)
    return problem, sims, masks, res


def train(data, epochs=20, batch=256, lr=1e-3, seed=0, device=0, log=None, tcgen05=True):
    """Adam with a short linear warm-up and a cosine decay; returns (net, losses per epoch)."""
    import torch
    H, Wd = data.n[1], data.n[2]
    net = U.UNet(batch, H, Wd, device=device, seed=seed, tcgen05=tcgen05)
    rng = np.random.default_rng(seed)
    nb = len(data) // batch
    losses = []
    total = epochs * nb
    k = 0
    for ep in range(epochs):
        perm_h = rng.permutation(len(data))[:nb * batch]
        perm = torch.tensor(perm_h, device=data.feats.device)
        acc = torch.zeros((), device=data.feats.device)
        for i in range(nb):
            idx = perm[i * batch:(i + 1) * batch]
            net.set_input(data.feats[idx])
            net.forward()
            net.set_target(data.targets[idx], data.masks[idx],
                           mask_count=data.mask_counts[perm_h[i * batch:(i + 1) * batch]].sum())
            acc += net.loss_and_grad()[0]
            net.backward()
            warm = min(1.0, (k + 1) / max(1, total // 20))
            net.adam(lr=lr * warm * 0.5 * (1 + np.cos(np.pi * k / total)))
            k += 1
        losses.append(float(acc.item()) / nb)
        net.check()
        if log:
            log(ep, losses[-1])
    return net, losses


def predict(net, sims, masks, n, host=False, mirror=True):
    """Initial states [nq][3N] (internal SoA, normalised, masked) for the problems, net.B
    per launch, built on the GPU from the problems' masks and parameters: a float32 device
    tensor (a host array with host=True).

    mirror=True also runs each problem's x-mirror image (Dataset's exact symmetry: mask
    reflected, u_y and B_y negated), maps that prediction back (reflected, m ->
    (m_x, -m_y, -m_z)) and averages the two before normalising: the network's errors on
    a problem and on its mirror image are partly independent."""
    import torch
    B = net.B
    nq = len(sims)
    ny, nx = n[1], n[2]
    P = ny * nx
    nqp = ((nq + B - 1) // B) * B
    mk = np.zeros((nqp, P), dtype=np.float32)
    mk[:nq] = np.stack(masks)
    prm = np.zeros((nqp, 8), dtype=np.float32)
    prm[:nq] = U.param_table(sims)
    mk_d = torch.tensor(mk, device=net.device)
    prm_d = torch.tensor(prm, device=net.device)
    out = torch.empty((nqp, 3 * P), dtype=torch.float32, device=net.device)
    if mirror:
        mk_m = torch.flip(mk_d.view(-1, ny, nx), dims=[2]).reshape(nqp, P).contiguous()
        prm_m = prm_d.clone()
        prm_m[:, U.PRM_AXIS_Y] *= -1.0
        prm_m[:, U.PRM_B_Y] *= -1.0
        tmp = torch.empty((B, 3 * P), dtype=torch.float32, device=net.device)
        sign = torch.tensor([-1.0, -1.0, 1.0], device=net.device).view(1, 3, 1, 1)   # internal (z, y, x)
    for i in range(0, nq, B):
        net.set_features(mk_d[i:i + B], prm_d[i:i + B])
        net.forward()
        net.states(mk_d[i:i + B], out[i:i + B])
        if mirror:
            net.set_features(mk_m[i:i + B], prm_m[i:i + B])
            net.forward()
            net.states(mk_m[i:i + B], tmp)
            back = torch.flip(tmp.view(B, 3, ny, nx), dims=[3]) * sign
            avg = out[i:i + B].view(B, 3, ny, nx) + back
            nrm = torch.sqrt((avg * avg).sum(dim=1, keepdim=True))
            avg = torch.where(nrm > 0, avg / nrm.clamp_min(1e-30), avg)
            out[i:i + B] = (avg * mk_d[i:i + B].view(B, 1, ny, nx)).reshape(B, 3 * P)
    net.check()
    out = out[:nq]
    return out.cpu().numpy() if host else out


def evaluate(net, problem, sims, masks, slots=256, device=0, energy_tol=1e-4, max_steps=20000, spec_frac=0.5,
             longest_first=True):
    """Cold and warm relaxations of the same problems (times include the network's
    inference for the warm start).  A warm relax that does not reach the threshold within
    max_steps (its step budget; step_budget() derives one from the training relaxations),
    or ends above the cold relax's energy by more than energy_tol (relative), counts as
    failed and is redone from the cold start in the same pool (time included).  The redo
    of a warm relax that has run spec_frac * max_steps steps starts beside it (relax_pool's
    spec_steps; 0 queues redos only once their warm relax is rejected).  Measured on 4096
    held-out problems: 0.05, 0.1, 0.25 and 0.5 of the budget gave 0.96, 1.09, 1.16 and
    1.18 times the cold rate (early redos take slots from the queue and are mostly
    cancelled).  longest_first: the warm pool starts its problems in decreasing order of the
    maxtorque / (gamma Ms) of their predicted start (computed in the timed region)."""
    import torch
    from .plan import Plan
    n = problem["n"]
    thr = thresholds(sims)
    cold = W.cold_state(n, 1)
    B = min(slots, len(sims))
    plan = Plan(problem, masks={"msat": np.concatenate(masks[:B])}, sims=sims[:B], masks_per_sim=True,
                device=device)
    if B > 16:   # the drain plan of both pools, made outside the timed regions
        _tail_plan(plan, problem, masks[0], sims[0], 16, device, 1e-6)
    # the problems' masks resident on the device for both pools (input data)
    masks_dev = torch.from_numpy(np.stack([np.asarray(m, dtype=np.float32) for m in masks])).to(
        plan.mask_tensor("msat").device)
    sims_arr = nat.make_sims(problem, sims)
    if longest_first:   # loads the tensor kernels of the ordering pass outside the timed regions
        initial_torques(plan, problem, sims[:1], masks[:1], None, masks_dev[:1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = relax_pool(problem, sims, masks, [cold] * len(sims), thr, slots=slots, device=device, plan=plan,
                    masks_dev=masks_dev)
    torch.cuda.synchronize()
    t_cold = time.perf_counter() - t0

    def accept(q, steps, mt, e):
        if not mt < thr[q]:
            return False
        return e <= rc["energy"][q] or abs(e - rc["energy"][q]) <= energy_tol * max(abs(rc["energy"][q]), 1e-30)

    t0 = time.perf_counter()
    init = predict(net, sims, masks, n)
    t0_warm = None
    order = None
    if longest_first:
        # the warm relaxations' lengths grow with the maxtorque of their start (about 130
        # steps per decade): start the problems in decreasing order of it
        t0_warm = initial_torques(plan, problem, sims, masks, init, masks_dev, sims_arr)
        order = np.argsort(-t0_warm, kind="stable")
    torch.cuda.synchronize()
    t_inf = time.perf_counter() - t0
    rw = relax_pool(problem, sims, masks, init, thr, slots=slots, device=device, max_steps=max_steps, plan=plan,
                    accept=accept, fallback=cold, spec_steps=int(spec_frac * max_steps), order=order,
                    masks_dev=masks_dev)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0
    # outside the timed regions: the maxtorque / (gamma Ms) of each start (cold and
    # predicted), one batched torque evaluation per slot group, against the steps taken
    if t0_warm is None:
        t0_warm = initial_torques(plan, problem, sims, masks, init, masks_dev, sims_arr)
    t0_cold = initial_torques(plan, problem, sims, masks, None, masks_dev, sims_arr)
    t = getattr(plan, "_tail_plan", None)
    if t is not None:
        t.close()
    plan.close()
    fb = rw["fell_back"]
    ok = ~fb
    lt = np.log10(np.maximum(t0_warm[ok], 1e-30))
    slope, icpt = np.polyfit(lt, rw["first_steps"][ok], 1) if ok.sum() > 2 else (float("nan"), float("nan"))
    erel = np.abs(rw["first_energy"] - rc["energy"]) / np.maximum(np.abs(rc["energy"]), 1e-30)
    return {
        "relaxations": len(sims),
        "cold_per_s": len(sims) / t_cold, "warm_per_s": len(sims) / t_warm,
        "speedup": t_cold / t_warm,
        "cold_steps_mean": float(rc["steps"].mean()), "warm_steps_mean": float(rw["first_steps"].mean()),
        "steps_saved_frac": float(1 - rw["first_steps"].sum() / max(1, rc["steps"].sum())),
        "warm_steps_incl_fallbacks_mean": float((rw["first_steps"] + np.where(fb, rw["steps"], 0)).mean()),
        "inference_s": t_inf, "warm_relax_only_per_s": len(sims) / (t_warm - t_inf),
        "warm_order": "decreasing initial maxtorque" if longest_first else "index",
        "cold_drive_s": rc["drive_s"], "cold_host_s": rc["host_s"], "warm_drive_s": rw["drive_s"],
        "warm_host_s": rw["host_s"],
        "cold_steps_max": int(rc["steps"].max()), "warm_steps_max": int(rw["first_steps"].max()),
        "warm_step_budget": int(max_steps),
        "warm_ok_frac": float(1 - fb.mean()), "fallbacks": int(fb.sum()),
        "spec_redos_started": int(rw["spec_started"]), "spec_redos_cancelled": int(rw["spec_cancelled"]),
        "final_converged_frac": float((rw["maxtorque"] < thr).mean()),
        "energy_within_tol_frac": float((erel <= energy_tol).mean()),
        "energy_rel_median": float(np.median(erel)),
        "warm_lower_energy_frac": float((rw["first_energy"] < rc["energy"]).mean()),
        "initial_torque_cold_median": float(np.median(t0_cold)),
        "initial_torque_warm_median": float(np.median(t0_warm)),
        "initial_torque_warm_p90": float(np.percentile(t0_warm, 90)),
        "warm_steps_vs_log10_initial_torque": {"slope": float(slope), "intercept": float(icpt),
                                               "fit_on": int(ok.sum())},
    }


def initial_torques(plan, problem, sims, masks, states, masks_dev=None, sims_arr=None):
    """maxtorque / (gamma Ms) of start states (a float32 device tensor [nq][3N], or the cold
    start when None), computed through the batched plan's torque, plan.nsim problems at a
    time (the plan's slots take their masks and scalars); one host read at the end.
    masks_dev: the problems' masks already on the device ([nq][N] float32), else they are
    uploaded here; sims_arr: their scalars as an mm_sim array (_native.make_sims)."""
    import ctypes as C

    import torch
    n = problem["n"]
    N = int(np.prod(n))
    B = plan.nsim
    nq = len(sims)
    mt = plan.mask_tensor("msat").view(-1, N)
    dev = mt.device
    if masks_dev is None:
        masks_dev = torch.from_numpy(np.stack([np.asarray(m, dtype=np.float32) for m in masks])).to(dev)
    if sims_arr is None:
        sims_arr = nat.make_sims(problem, sims)
    pad = nat.make_sims(problem, [sims[-1]] * B)   # fills the slots past the last problem
    cold = torch.tensor(W.cold_state(n, B), device=dev).view(-1) if states is None else None
    ms_all = torch.tensor([s["msat"] for s in sims], dtype=torch.float32, device=dev)
    out = torch.zeros(nq, dtype=torch.float32, device=dev)
    mbuf = torch.empty(3 * N * B, dtype=torch.float32, device=dev)
    tq = torch.empty(3 * N * B, dtype=torch.float32, device=dev)
    L = nat.lib()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    size = C.sizeof(nat.MMSim)
    for i in range(0, nq, B):
        k = min(B, nq - i)
        idx = torch.arange(i, i + B, device=dev).clamp(max=nq - 1)
        mt.copy_(masks_dev[idx])
        if k == B:
            nat.check(L.mm_batch_set_sims(plan.h, C.c_void_p(C.addressof(sims_arr) + i * size)))
        else:
            C.memmove(pad, C.addressof(sims_arr) + i * size, k * size)
            nat.check(L.mm_batch_set_sims(plan.h, C.cast(pad, C.c_void_p)))
        mbuf.copy_(cold if states is None else states[idx].reshape(-1))
        nat.check(L.mm_torque(plan.h, ptr(mbuf), 0, 0.0, ptr(tq), None))
        t3 = tq.view(B, 3, N)
        mx = torch.sqrt((t3 * t3).sum(dim=1)).max(dim=1).values
        out[i:i + k] = (mx / ms_all[idx])[:k]
    return out.cpu().numpy().astype(np.float64)
