"""The drop-in driver on a B200: the reference's prover.cpp, linked unchanged
against the library's C++ shim, runs the six families in the reference's order
(lane_packing.cu:32-37).  The test interrupts every family once with SIGINT
when its banner appears, so the interrupt takes effect after the family's
first launch over the whole lambda range (which holds failing boxes for every
family), and checks what the reference's SIGINT path prints
(run_kernel.cuh:86-108): the "We were interrupted" line, then the failing
boxes of that interval in the family's own line format (e.g.
middle_configuration.cu:182, end_configuration.cu:124,
start_configuration.cu:289).  Every launch is announced on stderr as
"Handling lambda interval [lb, ub]" (run_kernel.cuh:79).

When the reference-linked binary (oracle/_ref/prover_b200, built by
`make -C oracle ref`) is absent, the test builds the same three-line main from
its own source against the library."""
import os
import queue
import re
import signal
import subprocess
import threading
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "circlepacking_b200", "_lib")

MAIN = r"""
#include <cstddef>
namespace algcuda { namespace device { void set_printf_buffer_size(std::size_t); } }
namespace circlepacking { namespace lane_packing { extern void find_critical_intervals(); } }
int main() {
    algcuda::device::set_printf_buffer_size(64 * 1024 * 1024);
    circlepacking::lane_packing::find_critical_intervals();
    return 0;
}
"""

NUM = r"-?[0-9.]+(?:e[-+]?[0-9]+)?|inf|-inf|nan"
IV = rf"\[(?:{NUM}),(?:{NUM})\]"
# banner (stream, text) and (label prefix, separator, dims) of the critical lines, in the reference's order
FAMILIES = [
    (("out", "Start configuration..."), [("Critical interval: Start configuration, case 1", ": ", 4),
                                        ("Critical interval: Start configuration, case 2", ": ", 4)]),
    (("out", "Start & end configuration, 2 disks... "),
     [("Critical interval: Start & end configuration, 2 disks", ": ", 3)]),
    (("err", "Start & end configuration, 3 disks ..."), [("Start & end configuration: Critical interval", " - ", 4)]),
    (("out", "Middle configuration ..."), [("Critical interval: Middle configuration, case 1.1", ": ", 4),
                                           ("Critical interval: Middle configuration, case 2.1", ": ", 4)]),
    (("out", "End configuration (2 disks) ..."),
     [("End configuration (2 disks): Critical interval with r1 on the inside", " - ", 3),
      ("End configuration (2 disks): Critical interval with r1 on the outside", " - ", 3)]),
    (("out", "End configuration (3 disks) ..."),
     [("End configuration (3 disks): Critical interval with r1 on the inside", " - ", 4),
      ("End configuration (3 disks): Critical interval with r1 on the outside", " - ", 4)]),
]


def critical_re(label, sep, dims):
    axes = ["la", "r1", "r2", "r3"][:dims]
    return re.compile("^" + re.escape(label + sep) + ", ".join(f"{a} = {IV}" for a in axes) + "$")


def handling_line(lb, ub):
    """The reference's operator<< (interval.hpp:295-303): width 26, 19 digits."""
    return f"Handling lambda interval [{'%.19g' % lb:>26}, {'%.19g' % ub:>26}]"


def driver(tmp_path):
    prebuilt = os.path.join(ROOT, "oracle", "_ref", "prover_b200")
    if os.path.exists(prebuilt):
        return prebuilt
    src = tmp_path / "prover_main.cpp"
    src.write_text(MAIN)
    out = tmp_path / "prover_b200"
    subprocess.run(["g++", "-std=c++17", str(src), f"-L{LIBDIR}", "-lcp_b200", f"-Wl,-rpath,{LIBDIR}", "-o",
                    str(out)], check=True)
    return str(out)


def _pump(stream, tag, q):
    for line in iter(stream.readline, ""):
        q.put((tag, line.rstrip("\n")))
    q.put((tag, None))


@pytest.mark.gpu
def test_prover_sigint_prints_reference_format(cp, tmp_path):
    binary = driver(tmp_path)
    env = dict(os.environ, CP_CRITICALS_MAX="6")
    proc = subprocess.Popen([binary], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env,
                            start_new_session=True)
    q = queue.Queue()
    for s, tag in ((proc.stdout, "out"), (proc.stderr, "err")):
        threading.Thread(target=_pump, args=(s, tag, q), daemon=True).start()
    lines, open_streams = [], 2
    fam = -1             # family whose banner was seen last
    interrupted = set()  # families already sent their SIGINT
    deadline = time.monotonic() + 600
    try:
        while open_streams and time.monotonic() < deadline:
            try:
                tag, line = q.get(timeout=5)
            except queue.Empty:
                continue
            if line is None:
                open_streams -= 1
                continue
            lines.append((tag, line))
            for k, (banner, _) in enumerate(FAMILIES):
                if (tag, line) == banner and k not in interrupted:
                    fam = k
                    interrupted.add(k)
                    proc.send_signal(signal.SIGINT)
        rc = proc.wait(timeout=60)
    finally:
        if proc.poll() is None:
            os.killpg(proc.pid, signal.SIGKILL)
            proc.wait()
    text = "\n".join(f"{t}: {l}" for t, l in lines[-40:])
    assert rc == 0, f"driver exited {rc}:\n{text}"
    assert interrupted == set(range(6)), text
    # every family: its banner, the whole-domain first launch line, an interrupt
    # line, then its failing boxes in the reference's format.  stdout and stderr
    # are read by separate threads, so lines of the two streams may arrive out of
    # order: critical lines are attributed by their family label, not by position.
    handling = [l for t, l in lines if t == "err" and l.startswith("Handling lambda interval")]
    assert handling[0] == handling_line(0.5, 0.9900000000000001), handling[0]
    want_out = [b for (st, b), _ in FAMILIES if st == "out"]
    assert [l for t, l in lines if t == "out" and l in want_out] == want_out, text  # the reference's order
    interrupts = [l for t, l in lines
                  if t == "err" and l == "We were interrupted - running the first remaining interval with output once!"]
    assert len(interrupts) == 6, text
    crit = [l for t, l in lines if t == "out" and "Critical interval" in l]
    per_family = {k: 0 for k in range(6)}
    for l in crit:
        owners = [k for k, (_, labels) in enumerate(FAMILIES) if any(critical_re(*lab).match(l) for lab in labels)]
        assert len(owners) == 1, f"line not in any family's reference format: {l}"
        per_family[owners[0]] += 1
    for k, (banner, labels) in enumerate(FAMILIES):
        assert per_family[k] >= 1, f"{banner[1]}: no critical lines printed\n{text}"
        assert per_family[k] <= 6 * len(labels)
