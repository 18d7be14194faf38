"""Recipe that compiles the reference's own simulator kernels for parity checks (test
infrastructure).

Reads the reference's sources where they lie (the reference project root is taken from
$YB_REFERENCE_ROOT, default /root/reference) and writes only into oracle/_ref/:
  ref_nofma.fatbin   the kernels with every multiply and add rounded separately (-fmad=false),
                     the form the oracle's FP32 restatement must match bit for bit
  ref.fatbin         the kernels as the reference's own build compiles them (nvcc defaults,
                     contracted multiply-adds), for tolerance comparisons and timing
  libyb_ref.so       the host side (ref_host.cpp) that loads a fatbin and runs the schedule
When the reference is absent (as on the GPU machines) nothing is built and the files already in
oracle/_ref/ are used.  Nothing from the reference is copied into the repository.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"
CUDART_STATIC = "/usr/local/cuda/lib64/libcudart_static.a"

# the reference files the device build includes (relative to the reference's KittenEngine/)
REF_FILES = [
    "YarnBall/YarnBall.h", "YarnBall/YarnBall.cu", "YarnBall/sim/iteration.cu", "YarnBall/sim/collision.cu",
    "YarnBall/sim/cosserat.cu", "KittenEngine/includes/modules/Common.h", "KittenEngine/includes/modules/Rotor.h",
    "KittenEngine/includes/modules/SymMat.h", "KittenEngine/includes/modules/Bound.h",
]


def reference_root():
    return os.environ.get("YB_REFERENCE_ROOT", "/root/reference")


def _inputs(ke):
    own = []
    for dp, _, fs in os.walk(HERE):
        own += [os.path.join(dp, f) for f in fs if f.endswith((".h", ".hpp", ".cuh", ".cu", ".cpp"))]
    return own + [os.path.join(ke, f) for f in REF_FILES] + [os.path.join(ORACLE, "yb_oracle.h")]


def _stale(out, inputs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in inputs if os.path.exists(p))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def build(verbose=False):
    """Builds oracle/_ref when the reference is present; returns True if the outputs exist."""
    ke = os.path.join(reference_root(), "KittenEngine")
    outs = [os.path.join(OUT, f) for f in ("ref_nofma.fatbin", "ref.fatbin", "libyb_ref.so")]
    if not os.path.isdir(os.path.join(ke, "YarnBall")):
        return all(os.path.exists(o) for o in outs)
    os.makedirs(OUT, exist_ok=True)
    inputs = _inputs(ke)
    dev = os.path.join(HERE, "ref_device.cu")
    inc = ["-I", os.path.join(HERE, "inc"), "-I", ke]
    for fat, extra in ((outs[0], ["-fmad=false"]), (outs[1], [])):
        if _stale(fat, inputs):
            _run([NVCC, "-std=c++17", "-fatbin", "-gencode", "arch=compute_100a,code=sm_100a",
                  "-diag-suppress", "20012,177"] + extra + inc + [dev, "-o", fat])
            if verbose:
                sys.stderr.write("built %s\n" % fat)
    if _stale(outs[2], inputs):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-I", CUDA_INC,
              os.path.join(HERE, "ref_host.cpp"), "-o", outs[2], CUDART_STATIC, "-ldl", "-lrt", "-lpthread"])
    return True


if __name__ == "__main__":
    print(build(verbose=True))
