"""CPU-side checks of the C ABI (no GPU needed): the library loads, exports
every function include/sgfd.h declares, validates configurations before
touching a device, and fails cleanly when no device is present."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
import sgfd
import oracle_py


def header_functions():
    text = open(os.path.join(ROOT, "include", "sgfd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sgfd_\w+)\s*\(", text)))


def test_header_declares_api():
    names = header_functions()
    assert "sgfd_create" in names and "sgfd_step" in names and len(names) >= 20


def test_library_exports_every_declared_function():
    L = sgfd.lib()
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", sgfd.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sgfd_\w+)", out))
    assert set(header_functions()) <= exported


def test_abi_version_and_struct_size():
    assert sgfd.lib().sgfd_abi_version() == 1
    # int32 x4, float x4, float coef[5], int32, float, float, int32 x5, int32[7]
    assert ctypes.sizeof(sgfd.Config) == 4 * (4 + 4 + 5 + 3 + 5 + 7)


@pytest.mark.parametrize("kw,code", [
    (dict(pml=-1), sgfd.ERR_INVALID),
    (dict(nx=20, pml=10), sgfd.ERR_INVALID),
    (dict(dt=0.0), sgfd.ERR_INVALID),
    (dict(dx=-1.0), sgfd.ERR_INVALID),
    (dict(damping=7), sgfd.ERR_INVALID),
    (dict(quirks=3), sgfd.ERR_INVALID),
    (dict(damping=sgfd.DAMP_LOGR, damping_R=0.0), sgfd.ERR_INVALID),
    (dict(storage=9), sgfd.ERR_UNSUPPORTED),
    (dict(arith=5), sgfd.ERR_INVALID),
])
def test_create_rejects_bad_config(kw, code):
    cfg = sgfd.default_config(**kw)
    with pytest.raises(sgfd.SgfdError) as e:
        sgfd.Solver(cfg)
    assert e.value.code == code
    assert len(str(e.value)) > 20


def test_create_reports_missing_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(sgfd.SgfdError) as e:
        sgfd.Solver(sgfd.default_config())
    assert e.value.code == sgfd.ERR_NO_DEVICE


def test_ricker_matches_oracle_bitwise():
    for f0, dt in ((20.0, 0.0005), (25.0, 0.001), (2.0, 0.00175)):
        a = sgfd.ricker_ref(f0, dt, 600)
        b = oracle_py.ricker_ref(f0, dt, 600)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_pml_index_is_a_bijection(tmp_path):
    """Host-compiles the device layout helpers of csrc/sgfd_internal.h and checks
    that pml_index() maps the PML cells one-to-one onto [0, npml) for uneven
    sizes, and that the per-column/per-plane split the z-marching kernels use
    gives the same index."""
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include "sgfd_internal.h"
#include <cstdio>
#include <vector>
using namespace sgfd;
int main() {
  const int sizes[][4] = {{37,41,45,6},{23,23,23,1},{150,150,150,20},{60,33,41,3},{31,31,31,10}};
  for (auto &s : sizes) {
    Model m{}; m.nx=s[0]; m.ny=s[1]; m.nz=s[2]; m.pml=s[3];
    m.nxc=m.nx-10; m.nyc=m.ny-10; m.nzc=m.nz-10; m.px=m.nx; m.plane=(int64_t)m.px*m.ny;
    m.npml = pml_count(m.nxc, m.nyc, m.nzc, m.pml);
    std::vector<int> hit(m.npml, 0); int64_t cnt = 0;
    for (int z=5; z<m.nz-5; ++z) for (int y=5; y<m.ny-5; ++y) for (int x=5; x<m.nx-5; ++x) {
      int kx=band(x,m.nx,m.pml), ky=band(y,m.ny,m.pml), kz=band(z,m.nz,m.pml);
      if (!(kx|ky|kz)) continue;
      if (kx<0||kx>m.pml||ky<0||ky>m.pml||kz<0||kz>m.pml) { std::printf("bad band\n"); return 1; }
      int64_t i = pml_index(m, x-5, y-5, z-5);
      if (i < 0 || i >= m.npml) { std::printf("out of range %lld\n", (long long)i); return 1; }
      PmlColumn pc = pml_column(m, x-5, y-5);
      if (pml_plane_index(m, pc, z-5) != i) { std::printf("column/plane split differs\n"); return 1; }
      hit[i]++; cnt++;
    }
    if (cnt != m.npml) { std::printf("count %lld vs %lld\n", (long long)cnt, (long long)m.npml); return 1; }
    for (auto h : hit) if (h != 1) { std::printf("not bijective\n"); return 1; }
  }
  std::puts("ok"); return 0;
}
''')
    exe = tmp_path / "t"
    inc = os.path.join(ROOT, "staggered-grid_b200", "csrc")
    cuda_inc = "/usr/local/cuda/include"
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{inc}", f"-I{cuda_inc}", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
