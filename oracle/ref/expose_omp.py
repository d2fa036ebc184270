"""ORACLE — test infrastructure only.

Makes the OpenMP regions of the reference's main() callable by a harness.
GCC compiles every `#pragma omp parallel` block of ZebraflowWT.c's main() into
a local function `<main>._omp_fn.N`; this script finds, from the object's own
debug line table (built here with -g by oracle/ref/Makefile), the source line
of the `#pragma omp parallel` each one comes from, and writes a copy of the
object in which that function is a global symbol named zf_ref_omp_L<line>.

A harness then sets the reference's globals and calls a block as main() does
(GOMP_parallel(fn, data, 0, 0)): regions without shared locals take no data
(NULL); the few with shared locals take a struct of them.

Usage: python expose_omp.py <ZebraflowWT.c> <in.o> <out.o>
"""
import re
import shutil
import subprocess
import sys


def main():
    src, obj, out = sys.argv[1:4]
    lines = open(src, errors="replace").read().split("\n")
    syms = subprocess.run(["objdump", "-t", obj], check=True, capture_output=True, text=True).stdout
    ren = []
    for ln in syms.splitlines():
        m = re.match(r"^([0-9a-f]+)\s.*\s(\S+)\s+[0-9a-f]+\s+(\S+\._omp_fn\.\d+)$", ln)
        if not m:
            continue
        addr, sec, name = m.groups()
        where = subprocess.run(["addr2line", "-e", obj, "-j", sec, "0x" + addr], check=True,
                               capture_output=True, text=True).stdout.split()[0]
        line = int(where.rsplit(":", 1)[1].split()[0])
        # the pragma the region starts at: the nearest `#pragma omp parallel` at or above
        k = line
        while k > 0 and not re.match(r"\s*#pragma\s+omp\s+parallel", lines[k - 1]):
            k -= 1
        if k == 0:
            raise SystemExit(f"{name}: no `#pragma omp parallel` above line {line}")
        ren.append((name, f"zf_ref_omp_L{k}"))
    if len({b for _, b in ren}) != len(ren):
        raise SystemExit("two regions map to one pragma line")
    shutil.copyfile(obj, out)
    args = ["objcopy"]
    for a, b in ren:
        args += ["--redefine-sym", f"{a}={b}"]
    subprocess.run(args + [out], check=True)
    args = ["objcopy"]
    for _, b in ren:
        args += ["--globalize-symbol", b]
    subprocess.run(args + [out], check=True)
    for a, b in sorted(ren, key=lambda t: int(t[1].rsplit("L", 1)[1])):
        print(f"{b} <- {a}")


if __name__ == "__main__":
    main()
