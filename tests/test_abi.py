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
    sizes, that the per-column/per-plane split the z-marching kernels use
    gives the same index, and that the blocked split storage (split k of cell
    c at split_base(c) + 32 k) gives every (cell, split) its own value inside
    split_elems(npml), in 64-bit and 32-bit form.  Then cuts each model into
    z-slabs: a slab's z bands, compact indices (whole-model index minus the
    slab's base, in both forms) and PML count agree with the whole model's."""
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
    m.nzcg = m.nzc;
    m.npml = pml_count(m.nxc, m.nyc, m.nzc, m.pml);
    if (pml_before(m.nxc, m.nyc, m.nzc, m.pml, m.nzc) != m.npml) { std::printf("pml_before\n"); return 1; }
    std::vector<int> hit(m.npml, 0); int64_t cnt = 0;
    for (int z=5; z<m.nz-5; ++z) for (int y=5; y<m.ny-5; ++y) for (int x=5; x<m.nx-5; ++x) {
      int kx=band(x,m.nx,m.pml), ky=band(y,m.ny,m.pml), kz=bandz(m,z);
      if (kz != band(z,m.nz,m.pml)) { std::printf("bandz\n"); return 1; }
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
    std::vector<unsigned char> used(split_elems(m.npml), 0);
    for (int64_t c = 0; c < m.npml; ++c)
      for (int k = 0; k < kNumSplit; ++k) {
        const int64_t j = split_base(c) + (int64_t)k * kSplitBlock;
        if (j < 0 || j >= (int64_t)used.size() || used[j]++) { std::printf("split slot %lld\n", (long long)j); return 1; }
        if ((int64_t)split_base32((uint32_t)c) != split_base(c) || split_of(j) != k) { std::printf("split forms\n"); return 1; }
      }
    // z-slabs at uneven cuts (1-plane slabs included)
    const int nzc = m.nzc;
    const int cutsets[3][3] = {{nzc / 3, 2 * nzc / 3, nzc}, {1, nzc - 1, nzc}, {m.pml, m.pml + 1, nzc}};
    for (auto &cs : cutsets) {
      int64_t total = 0; int z0 = 0;
      for (int e : cs) {
        if (e <= z0) continue;
        Model q = m; q.nz = (e - z0) + 10; q.nzc = e - z0; q.zoff = z0; q.nzcg = nzc;
        q.pbase = pml_before(m.nxc, m.nyc, nzc, m.pml, z0);
        q.npml = pml_before(m.nxc, m.nyc, nzc, m.pml, e) - q.pbase;
        int64_t c2 = 0;
        for (int z=5; z<q.nz-5; ++z) for (int y=5; y<m.ny-5; ++y) for (int x=5; x<m.nx-5; ++x) {
          const int kz = bandz(q, z);
          if (kz != band(z + z0, m.nz, m.pml)) { std::printf("slab band\n"); return 1; }
          if (!(band(x,m.nx,m.pml) | band(y,m.ny,m.pml) | kz)) continue;
          const int64_t i = pml_index(q, x-5, y-5, z-5);
          if (i != pml_index(m, x-5, y-5, z-5+z0) - q.pbase || i < 0 || i >= q.npml) { std::printf("slab index\n"); return 1; }
          if (pml_plane_index(q, pml_column(q, x-5, y-5), z-5) != (uint32_t)i) { std::printf("slab plane index\n"); return 1; }
          ++c2;
        }
        if (c2 != q.npml) { std::printf("slab count\n"); return 1; }
        total += q.npml; z0 = e;
      }
      if (total != m.npml) { std::printf("slab total\n"); return 1; }
    }
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


def test_half_step_parts_cover_every_unit_once(tmp_path):
    """Host-compiles part_ranges() of csrc/sgfd_internal.h, which splits a half
    step into the units (z chunks, or planes) a z-slab runs while its halos
    travel and the rest: for every plane count and unit size, the inner and
    outer parts together cover each unit exactly once, an inner unit's planes
    lie 5 or more planes from both ends (its updates read no frame plane),
    every outer unit has a plane closer than that, and the whole half step
    is one range."""
    src = tmp_path / "p.cpp"
    src.write_text(r'''
#include "sgfd_internal.h"
#include <cstdio>
#include <vector>
using namespace sgfd;
int main() {
  for (int nzc = 1; nzc <= 130; ++nzc)
    for (int size = 1; size <= 60; ++size) {
      const int n = (nzc + size - 1) / size;
      int r[3][2];
      if (part_ranges(nzc, size, n, kPartInner | kPartOuter, r) != 1 || r[0][0] != 0 || r[0][1] != n) {
        std::printf("whole %d %d\n", nzc, size); return 1;
      }
      std::vector<int> seen(n, 0);
      for (int part : {kPartInner, kPartOuter}) {
        const int k = part_ranges(nzc, size, n, part, r);
        int prev = 0;
        for (int i = 0; i < k; ++i) {
          if (r[i][0] < prev || r[i][1] < r[i][0] || r[i][1] > n) { std::printf("order %d %d\n", nzc, size); return 1; }
          prev = r[i][1];
          for (int u = r[i][0]; u < r[i][1]; ++u) {
            const int zs = u * size, ze = (u + 1) * size < nzc ? (u + 1) * size : nzc;
            const bool inner = zs >= kHalo && ze <= nzc - kHalo;
            if (inner != (part == kPartInner)) { std::printf("unit %d of %d %d\n", u, nzc, size); return 1; }
            seen[u]++;
          }
        }
      }
      for (int u = 0; u < n; ++u) if (seen[u] != 1) { std::printf("cover %d %d\n", nzc, size); return 1; }
    }
  std::puts("ok"); return 0;
}
''')
    exe = tmp_path / "p"
    inc = os.path.join(ROOT, "staggered-grid_b200", "csrc")
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{inc}", "-I/usr/local/cuda/include", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout


def test_strip_tiles_cover_the_strip_once(tmp_path):
    """Host-compiles csrc/strip_tiles.h and checks the learned strip's tiling
    for uneven sizes and widths: every strip cell in exactly one tile, no
    interior cell in any, every box within 128 cells and its one-cell halo
    within the 544 staged cells; and the staging index split of k_strip_tc
    (quotients through a float reciprocal) equal to integer division for every
    staged cell of every box."""
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include "strip_tiles.h"
#include <cstdio>
#include <vector>
using namespace sgfd;
int main() {
  const int cases[][4] = {{20,20,20,6},{268,268,268,6},{58,47,63,6},{30,31,29,1},{40,40,40,3},
                          {100,90,80,33},{21,22,23,10},{70,70,70,2},{90,91,92,16},{200,150,120,12}};
  for (auto &c : cases) {
    const int X = c[0], Y = c[1], Z = c[2], w = c[3];
    std::vector<int4> t;
    if (strip_tiles(X, Y, Z, w, t) != (int)t.size()) { std::printf("does not fit\n"); return 1; }
    std::vector<int> hit((size_t)X * Y * Z, 0);
    for (auto &q : t) {
      const int ex = q.w & 255, ey = (q.w >> 8) & 255, ez = (q.w >> 16) & 255;
      if (ex < 1 || ey < 1 || ez < 1 || ex * ey * ez > kStripRows) { std::printf("bad extents\n"); return 1; }
      if ((ex + 2) * (ey + 2) * (ez + 2) > kStripStage) { std::printf("halo too large\n"); return 1; }
      if (q.x < 0 || q.y < 0 || q.z < 0 || q.x + ex > X || q.y + ey > Y || q.z + ez > Z) { std::printf("outside\n"); return 1; }
      for (int z = q.z; z < q.z + ez; ++z) for (int y = q.y; y < q.y + ey; ++y) for (int x = q.x; x < q.x + ex; ++x)
        hit[((size_t)z * Y + y) * X + x]++;
      const int sx = ex + 2, sxy = sx * (ey + 2), ns = sxy * (ez + 2);
      const float inv_sx = 1.0f / (float)sx, inv_sxy = 1.0f / (float)sxy;
      for (int r = 0; r < ns; ++r) {
        const int lz = (int)(((float)r + 0.5f) * inv_sxy), rr = r - lz * sxy;
        const int ly = (int)(((float)rr + 0.5f) * inv_sx), lx = rr - ly * sx;
        if (lz != r / sxy || ly != (r % sxy) / sx || lx != r % sx) { std::printf("staging index\n"); return 1; }
      }
    }
    for (int z = 0; z < Z; ++z) for (int y = 0; y < Y; ++y) for (int x = 0; x < X; ++x) {
      const bool strip = x < w || y < w || z < w || x >= X - w || y >= Y - w || z >= Z - w;
      if (hit[((size_t)z * Y + y) * X + x] != (strip ? 1 : 0)) { std::printf("cover\n"); return 1; }
    }
  }
  std::puts("ok"); return 0;
}
''')
    exe = tmp_path / "t"
    inc = os.path.join(ROOT, "staggered-grid_b200", "csrc")
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{inc}", "-I/usr/local/cuda/include", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout


def test_entry_points_reject_a_null_handle():
    """Without a handle the stepping, halo and medium calls return
    SGFD_ERR_INVALID instead of touching a device (their profiler trace
    ranges open and close on the host all the same)."""
    L = sgfd.lib()
    assert L.sgfd_run(None, 0, 1, 0) == sgfd.ERR_INVALID
    assert L.sgfd_step(None, 0, 0.0) == sgfd.ERR_INVALID
    assert L.sgfd_step_phase(None, 0, 0.0, sgfd.PHASE_VELOCITY) == sgfd.ERR_INVALID
    assert L.sgfd_step_phase_part(None, 0, 0.0, sgfd.PHASE_STRESS, sgfd.PART_INNER) == sgfd.ERR_INVALID
    assert L.sgfd_halo_pack(None, sgfd.HALO_LOW, sgfd.HALO_STRESS, None) == sgfd.ERR_INVALID
    assert L.sgfd_halo_unpack(None, sgfd.HALO_HIGH, sgfd.HALO_VELOCITY, None) == sgfd.ERR_INVALID
    n = ctypes.c_int64(-1)
    assert L.sgfd_halo_bytes(None, ctypes.byref(n)) == sgfd.ERR_INVALID
    assert L.sgfd_set_medium(None, None, None, None) == sgfd.ERR_INVALID
