"""The multi-GPU path of bench.py on CPUs: N independent replicas with a
barrier around the timed region, the slowest rank's time and the aggregate
rate (sph-2d_b200/replicas.py), here as two gloo ranks that each advance the
oracle; and the reference arm's rule that only rank 0 works."""
import os
import socket
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "sph-2d_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_api as O
    import replicas
    import sph_b200 as S
    r, w, _ = replicas.dist_env()
    replicas.init(w, "gloo", timeout_s=60)
    case = S.make_tgv(16, solver=S.SOLVER_MODLR_DELTA_SPS)
    sim = O.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
    replicas.barrier(w)
    t0 = time.perf_counter()
    sim.run(2, S.baseline_dt(case.cfg))
    if r == 1:
        time.sleep(0.3)          # the slow replica
    el = time.perf_counter() - t0
    replicas.barrier(w)
    mx = replicas.max_over_ranks(el, w)
    rate = replicas.aggregate_rate(case.n * 2, w, mx)
    q.put((r, el, mx, rate, case.n, sim.kinetic_energy()))
    replicas.shutdown(w)


def test_two_gloo_replicas_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, el0, mx0, rate0, n, ke0), (r1, el1, mx1, rate1, _, ke1) = out
    assert (r0, r1) == (0, 1)
    assert mx0 == mx1 == max(el0, el1) and mx1 >= 0.3
    assert rate0 == rate1 == 2 * n * 2 / mx0
    assert ke0 == ke1                      # identical, independent replicas


def test_reference_arm_works_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"], env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
