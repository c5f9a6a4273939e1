"""The FP32 method keeps its x-slab CPML integrators in rows aligned to the
4-cell groups (Slab::lo4 in fdtd_b200/csrc/internal.h); the layout functions
the kernels and the host read-back share are checked on the CPU for every
axis length 6..300 and CPML widths 0..20 at each end
(tests/cpp/xslab_layout_check.cu)."""
import os
import subprocess

from fdtd_b200.build_lib import NVCC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_aligned_x_slab_layout(tmp_path):
    exe = str(tmp_path / "xslab_layout_check")
    subprocess.run([NVCC, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "xslab_layout_check.cu")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "layouts checked" in out.stdout
