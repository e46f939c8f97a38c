"""Build recipe for the oracle (TEST INFRASTRUCTURE ONLY).

* oracle/_build/libsrk_oracle.so  — the FP64 C restatement (srk_oracle.c), gcc.
* oracle/_ref/libref_host.so      — the reference's own host generators
  (GpGenerator, generate_pattern) compiled from its sources, nvcc host code.
* oracle/_ref/libref_gpu.so       — the reference's own srkTrainingForward and
  MeasureCD_Batched compiled for sm_100a from its sources (cuFFT, Thrust).

The reference builds need the reference sources, so they are only built where
those exist; the built files travel with the repository snapshot.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# The reference checkout: $SRK_REFERENCE_DIR, else a directory named
# "reference" beside the repository (the checkout layout this recipe is
# used with).  Nothing is built from it when neither exists.
REF_SRC = os.environ.get("SRK_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "srk_oracle.c")
    out = os.path.join(BUILD, "libsrk_oracle.so")
    if force or _stale(out, [src]):
        _run(["gcc", "-O3", "-march=x86-64-v2", "-fPIC", "-shared", "-std=c11", "-D_GNU_SOURCE",
              src, "-o", out, "-lm", "-lpthread"])
    return out


def build_reference(force=False):
    """Compile the reference's host generators and GPU training forward."""
    if not os.path.isdir(REF_SRC):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    inc = os.path.join(REF_SRC, "third_party", "include")
    host_src = [os.path.join(HERE, "ref_wrap", "ref_host.cpp"),
                os.path.join(REF_SRC, "third_party", "src", "patternUtil", "test_pattern.cu")]
    host_out = os.path.join(REF_OUT, "libref_host.so")
    if force or _stale(host_out, host_src):
        _run([NVCC, "-std=c++17", "-O2", "-x", "cu"] + ARCH +
             ["-Xcompiler", "-fPIC", "-shared", "-I" + inc] + host_src + ["-o", host_out])
    gpu_src = [os.path.join(HERE, "ref_wrap", "ref_gpu.cu"),
               os.path.join(REF_SRC, "third_party", "src", "metricUtil", "cd_measure_util.cu")]
    gpu_out = os.path.join(REF_OUT, "libref_gpu.so")
    if force or _stale(gpu_out, gpu_src):
        _run([NVCC, "-std=c++17", "-O2", "--extended-lambda"] + ARCH +
             ["-Xcompiler", "-fPIC", "-shared", "-I" + inc, "-I" + os.path.join(REF_SRC, "training")] +
             gpu_src + ["-lcufft", "-lcudnn", "-o", gpu_out])
    return REF_OUT


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
