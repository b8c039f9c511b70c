"""The tcgen05 operand layout and descriptors of firtez-dz_b200/csrc/fz_tc.cuh,
checked on the CPU before any of it runs on a GPU.

A host program including the header (compiled by nvcc, run on the CPU)
prints the packed instruction and shared-memory descriptors and the byte
offsets the Gram kernel stores its bf16 operands at.  They are compared
with the field layout of the tcgen05 descriptors (PTX ISA; the same fields
CUTLASS's UMMA::InstrDescriptor and SmemDescriptor name): instruction
descriptor -- D format F32 at bits 4-5, A and B format BF16 at 7-9 and
10-12, K-major A and B (bits 15, 16 zero), N >> 3 at 17-22, M >> 4 at
24-28; shared-memory descriptor -- start address >> 4 at 0-13, LBO >> 4 at
16-29, SBO >> 4 at 32-45, version 1 at 46, no swizzle (61-63 zero).  The
operand offsets must tile a 128 x 64 bf16 tile without overlap inside its
16 KB, in 8-byte aligned runs of four K elements, and agree with the
canonical K-major no-swizzle addressing each MMA's descriptor implies:
element (r, k) of the 16-wide K step ks at start + (r % 8) * 16 + (r / 8) *
SBO + (k % 8) * 2 + (k / 8) * LBO with start = 256 ks, LBO = 128, SBO = 1024.
The tile-pair decoding of the Gram kernel covers every block pair once.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("tc")
    src = d / "probe.cu"
    src.write_text(r'''
#include <cstdio>
#include "fz_tc.cuh"
int main() {
  for (int n = 16; n <= 128; n += 16) std::printf("I %d %u\n", n, fztc::idesc_bf16(128, n));
  std::printf("S %llu\n", (unsigned long long)fztc::desc_kmajor(0x1230u, 128u, 1024u));
  std::printf("W %llu\n", (unsigned long long)fztc::desc_sw128(0x4c00u + 32u));
  std::printf("M %llu\n", (unsigned long long)fztc::desc_sw128_mn(0x4c00u + 2048u, 8192u));
  std::printf("J %u %u %u\n", fztc::idesc_bf16_major(128, 128, false, true), fztc::idesc_bf16_major(128, 128, true, true),
              fztc::idesc_bf16(128, 128));
  for (int r = 0; r < 128; ++r)
    for (int k = 0; k < 64; k += 4) std::printf("O %d %d %u\n", r, k, fztc::kmajor_offset(r, k, 8));
  return 0;
}
''')
    exe = d / "probe"
    subprocess.check_call([NVCC, "-std=c++17", "-arch=sm_100a", "-I", os.path.join(ROOT, "firtez-dz_b200", "csrc"),
                           str(src), "-o", str(exe)])
    return subprocess.check_output([str(exe)]).decode().split("\n")


def field(v, lo, n):
    return (v >> lo) & ((1 << n) - 1)


def test_instruction_descriptor(probe):
    for ln in probe:
        if ln.startswith("I "):
            _, n, v = ln.split()
            n, v = int(n), int(v)
            assert field(v, 0, 4) == 0                       # dense, no saturate
            assert field(v, 4, 2) == 1                       # D: F32
            assert field(v, 7, 3) == 1 and field(v, 10, 3) == 1   # A, B: BF16
            assert field(v, 13, 2) == 0                      # no negation
            assert field(v, 15, 1) == 0 and field(v, 16, 1) == 0  # K-major A and B
            assert field(v, 17, 6) == n >> 3 and field(v, 24, 5) == 128 >> 4
            assert field(v, 23, 1) == 0 and field(v, 29, 3) == 0


def test_shared_memory_descriptor(probe):
    v = int([ln for ln in probe if ln.startswith("S ")][0].split()[1])
    assert field(v, 0, 14) == 0x1230 >> 4
    assert field(v, 16, 14) == 128 >> 4
    assert field(v, 32, 14) == 1024 >> 4
    assert field(v, 46, 2) == 1                              # Blackwell descriptor version
    assert field(v, 49, 3) == 0 and field(v, 52, 1) == 0    # base offset, LBO mode
    assert field(v, 61, 3) == 0                              # SWIZZLE_NONE


def test_swizzled_shared_memory_descriptor(probe):
    """The descriptor of the TMA-fed GEMM's tiles: K-major, 128-byte
    swizzle (layout type 2), 8-row groups 1 KB apart, LBO unused, the start
    address of a 1 KB-aligned tile advanced by 32 B for the second K step."""
    v = int([ln for ln in probe if ln.startswith("W ")][0].split()[1])
    assert field(v, 0, 14) == (0x4c00 + 32) >> 4
    assert field(v, 16, 14) == 0
    assert field(v, 32, 14) == 1024 >> 4
    assert field(v, 46, 2) == 1
    assert field(v, 49, 3) == 0 and field(v, 52, 1) == 0
    assert field(v, 61, 3) == 2                              # SWIZZLE_128B


def test_mn_major_descriptors(probe):
    """MN-major operands of the backward GEMMs: the 128-byte-swizzled tile of
    two 64-element MN halves 8 KB apart (LBO) with 8-row K groups 1 KB apart
    (SBO), the start advanced 2 KB per 16-wide K step; the instruction
    descriptor's A- and B-major bits (15, 16) set for MN-major operands,
    nothing else changed."""
    v = int([ln for ln in probe if ln.startswith("M ")][0].split()[1])
    assert field(v, 0, 14) == (0x4c00 + 2048) >> 4
    assert field(v, 16, 14) == 8192 >> 4
    assert field(v, 32, 14) == 1024 >> 4
    assert field(v, 46, 2) == 1 and field(v, 61, 3) == 2
    b_mn, ab_mn, plain = (int(x) for x in [ln for ln in probe if ln.startswith("J ")][0].split()[1:])
    assert b_mn == plain | (1 << 16) and ab_mn == plain | (1 << 15) | (1 << 16)


def test_operand_offsets_match_the_descriptor_addressing(probe):
    offs = {}
    for ln in probe:
        if ln.startswith("O "):
            _, r, k, o = ln.split()
            offs[(int(r), int(k))] = int(o)
    assert len(offs) == 128 * 16
    seen = set()
    for (r, k), o in offs.items():
        assert o % 8 == 0 and 0 <= o and o + 8 <= 128 * 64 * 2
        for e in range(4):                                   # four consecutive K elements, 2 bytes each
            seen.add(o + 2 * e)
            kk = k + e
            ks, kw = kk // 16, kk % 16
            canon = 256 * ks + (r % 8) * 16 + (r // 8) * 1024 + (kw % 8) * 2 + (kw // 8) * 128
            assert o + 2 * e == canon, (r, kk)
    assert len(seen) == 128 * 64                             # no two elements share a byte pair


@pytest.mark.parametrize("npar", [17, 128, 129, 300, 512, 1024])
def test_gram_tile_pairs_cover_the_matrix(npar):
    """The Gram kernel's grid (nb (nb + 1) / 2 tile pairs) decodes into every
    block pair bi <= bj exactly once, rows and columns inside np."""
    nb = (npar + 127) // 128
    pairs = []
    for b in range(nb * (nb + 1) // 2):
        t, bi = b, 0
        while bi < nb and t >= nb - bi:
            t -= nb - bi
            bi += 1
        assert bi < nb
        pairs.append((bi, bi + t))
    assert sorted(pairs) == [(i, j) for i in range(nb) for j in range(i, nb)]
    for bi, bj in pairs:
        n = min(128, npar - bj * 128)
        assert 0 < n <= 128 and ((n + 15) & ~15) <= 128
