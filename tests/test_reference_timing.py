"""oracle/time_reference_build.py (the timing of the reference's own CUDA build) on a stand-in
executable that writes the per-step log the reference-build hooks write (step, dt,
n_leaves, wall_s since start; oracle/ref/hooks.cu): ms per step and updates/s come from the
steps after the warm-up only, and the run is stopped after warm-up + timed steps."""
import json
import os
import stat
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAKE = """#!{py}
import os
n = int(os.environ["MWDG2_REF_STOP_AFTER"])
with open(os.environ["MWDG2_REF_STEPS_CSV"], "w") as f:
    f.write("step,dt,n_leaves,wall_s\\n")
    for s in range(1, n + 1):
        f.write(f"{{s}},0.1,{{1000 + s}},{{2.0 + 0.004 * s + (0.5 if s == 1 else 0.0):.9f}}\\n")
"""


def test_reference_timing_uses_the_steps_after_the_warmup(tmp_path):
    exe = tmp_path / "fake_ref"
    exe.write_text(FAKE.format(py=sys.executable))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "time_reference_build.py"), "--level", "7",
                        "--steps", "4", "--warmup", "2", "--case-dir", str(tmp_path / "cases"), "--exe", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    # steps 3..6: leaves 1003..1006, 4 ms apart (the slow first step is warm-up)
    assert d["steps"] == 4 and d["warmup"] == 2
    assert abs(d["ms_per_step"] - 4.0) < 1e-6
    assert abs(d["leaves_mean"] - 1004.5) < 1e-9
    assert abs(d["value"] - 4018 / 0.016) < 1e-3


FAKE_WINDOW = """#!{py}
import os
T = float(os.environ["MWDG2_REF_WINDOW_TIME"])
n = int(os.environ["MWDG2_REF_WINDOW_STEPS"])
first = None
with open(os.environ["MWDG2_REF_STEPS_CSV"], "w") as f:
    f.write("step,dt,n_leaves,wall_s,time\\n")
    t, s = 0.0, 0
    while True:
        s += 1
        t += 0.5
        f.write(f"{{s}},0.5,{{100 * s}},{{0.01 * s:.9f}},{{t:.9f}}\\n")
        if first is None and t >= T:
            first = s
        if first is not None and s >= first + n:
            break
"""


def test_reference_timing_window_later_in_the_run(tmp_path):
    """A window from simulated time T: the steps after the first one that ends at t >= T,
    W of them untimed, then K timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import time_reference_build
    exe = tmp_path / "fake_ref"
    exe.write_text(FAKE_WINDOW.format(py=sys.executable))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    par = tmp_path / "case.par"
    par.write_text("mwdg2\n")
    d = time_reference_build.time_reference(str(par), 32, steps=4, warmup=2, exe=str(exe), window_time=10.0)
    # t = 0.5 s per step: step 20 ends at t = 10; warm-up steps 21, 22; timed steps 23..26
    assert d["window"]["first_step"] == 23
    assert abs(d["ms_per_step"] - 10.0) < 1e-6
    assert abs(d["leaves_mean"] - 2450.0) < 1e-9
    assert abs(d["wall_s_per_sim_s"] - 0.04 / 2.0) < 1e-9
