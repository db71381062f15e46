"""Host-side pieces of the benchmark, on the CPU: the core count of the CPU baseline and the
device-side generator of the realistic records (run here with torch on the CPU)."""
import os
import subprocess
import sys
import textwrap

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_core_count_survives_an_openmp_region():
    """With OMP_PROC_BIND set, the first OpenMP region binds the calling thread to one place;
    the benchmark counts its cores from the affinity mask it read at start, so the count after
    the oracle has run (the CPU baseline's own OpenMP region) is the count before it."""
    script = textwrap.dedent(f"""
        import os, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        before = bench.physical_cores()
        from oracle import bindings as ob
        from wacommplusplus_b200 import synthetic as syn
        from wacommplusplus_b200.types import default_config
        win = syn.config1_window(n_frames=2, eta=16, xi=16, s_rho=4)
        p = syn.uniform_particles(256, win.eta, win.xi, seed=1)
        ob.oracle_move(default_config(random=False), p, win, 0, ob.SEMANTICS_HOST, threads=2)
        after = bench.physical_cores()
        print(before[0], after[0], len(bench.CPU_SET))
    """)
    env = dict(os.environ, OMP_PROC_BIND="close", OMP_PLACES="cores")
    out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, env=env,
                         check=True, timeout=300).stdout.split()
    before, after, cpus = (int(x) for x in out[-3:])
    assert before == after >= 1
    assert cpus == len(os.sched_getaffinity(0))


def test_realistic_records_from_the_device_generator():
    """frame_device reproduces frame's streamfunction velocities and surface elevation; its w
    and AKT noise (torch's seeded generator) has the distribution frame draws from and repeats
    for the same record."""
    from wacommplusplus_b200 import synthetic as syn
    forcing = syn.RealisticForcing(eta=96, xi=80, s_rho=10, n_frames=3, seed=21)
    host = forcing.frame(1)
    dev = forcing.frame_device(1, "cpu")
    for key in ("zeta", "u", "v"):
        assert dev[key].dtype == np.float32 and dev[key].shape == host[key].shape
        assert np.allclose(dev[key], host[key], rtol=1e-6, atol=1e-7), key
    water = forcing.water
    w = dev["w"][:, water]
    assert abs(w.mean()) < 5e-6 and abs(w.std() / 1e-4 - 1.0) < 0.05
    log_akt = np.log(dev["akt"][:, water] / 1e-4)
    assert abs(log_akt.mean()) < 0.05 and abs(log_akt.std() - 1.0) < 0.05
    assert not dev["w"][:, ~water].any() and not dev["akt"][:, ~water].any()
    again = forcing.frame_device(1, "cpu")
    assert np.array_equal(again["w"], dev["w"]) and np.array_equal(again["akt"], dev["akt"])
    win = forcing.window_of([1], [dev])
    assert win.u.shape == (1,) + host["u"].shape and win.times[0] == forcing.times[1]
