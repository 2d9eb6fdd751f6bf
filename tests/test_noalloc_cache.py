"""The address cache behind octo_beam_gaussian_noalloc, on the CPU.

The allocation-free entry point passes its kernels the device address of a static scratch array.  That
address belongs to the module loaded in the device's current context; after a device reset a new context
loads the module again, possibly elsewhere, so the cache (octopus.jl_b200/csrc/noalloc_cache.h) keys each
device's address by the context it was looked up in.  This test compiles the header with the host compiler
and drives it with fake context handles and a counting resolver: same context -> no new lookup; new
context on the same device -> a new lookup and the new address; devices independent; a failed lookup is
not cached; out-of-range devices rejected."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "octopus.jl_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "noalloc_cache.h"

#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d: %s\n", __LINE__, #c); return 1; } } while (0)

int main() {
    octo::SymbolAddressCache<4> cache;
    int ctxA = 0, ctxB = 0;  // stand-ins for two driver context handles
    char module1[8], module2[8], module3[8];
    int resolves = 0;
    void *next = module1;
    auto resolve = [&]() -> void * { ++resolves; return next; };

    CHECK(cache.lookup(0, &ctxA, resolve) == module1);   // first call: looked up
    CHECK(resolves == 1);
    next = module2;
    CHECK(cache.lookup(0, &ctxA, resolve) == module1);   // same context: cached, not looked up
    CHECK(resolves == 1);
    CHECK(cache.lookup(0, &ctxB, resolve) == module2);   // context changed (device reset): looked up again
    CHECK(resolves == 2);
    CHECK(cache.lookup(0, &ctxB, resolve) == module2);
    CHECK(resolves == 2);
    next = module3;
    CHECK(cache.lookup(1, &ctxA, resolve) == module3);   // another device: its own slot
    CHECK(resolves == 3);
    CHECK(cache.lookup(0, &ctxB, resolve) == module2);   // device 0 unaffected
    next = nullptr;
    CHECK(cache.lookup(2, &ctxA, resolve) == nullptr);   // failed lookup: reported, not cached
    CHECK(resolves == 4);
    next = module1;
    CHECK(cache.lookup(2, &ctxA, resolve) == module1);   // retried on the next call
    CHECK(resolves == 5);
    CHECK(cache.lookup(-1, &ctxA, resolve) == nullptr);  // out of range: no lookup
    CHECK(cache.lookup(4, &ctxA, resolve) == nullptr);
    CHECK(resolves == 5);
    CHECK(cache.lookups() == 4);
    std::printf("ok\n");
    return 0;
}
"""


def test_address_cache_is_invalidated_when_the_context_changes(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "cache_driver.cpp"
    exe = tmp_path / "cache_driver"
    src.write_text(DRIVER)
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", HEADER_DIR, str(src), "-o", str(exe), "-pthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
