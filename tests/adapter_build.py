"""Builds the adapter parity program (tests/adapter_parity.cc) into
tests/_bin/adapter_parity against the reference's own MobBase / BrwnBase /
ForceBase headers and base-class sources, where they lie in the reference
tree (nothing is copied out of it).  Test infrastructure: called by
tests/test_adapters.py and __graft_entry__.build() where the reference tree is
present; the GPU test runs the prebuilt program."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(HERE, "_bin", "adapter_parity")


def compile_cmd(ref: str, src: str, exe: str) -> list:
    """g++ line for a translation unit that includes the adapters and the
    reference's base-class headers (gnu++98, as the reference)."""
    extra = [os.path.join(ref, "src", "mob", "mob_base.cc"), os.path.join(ref, "src", "brwn", "brwn_base.cc"),
             os.path.join(ref, "src", "force", "force_base.cc")]
    lib = os.path.join(ROOT, "stokesdt_b200")
    return (["g++", "-O2", "-std=gnu++98", "-D__declspec(a)=__attribute__((aligned(64)))",
             "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ref, "src", "mob"),
             "-I", os.path.join(ref, "src", "brwn"), "-I", os.path.join(ref, "src", "util"),
             "-I", os.path.join(ref, "src", "force"), src] + extra +
            ["-o", exe, "-L", lib, "-l:libstokesdt_b200.so", "-Wl,-rpath,$ORIGIN/../../stokesdt_b200"])


def build(ref: str) -> str:
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    res = subprocess.run(compile_cmd(ref, os.path.join(HERE, "adapter_parity.cc"), BIN),
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"adapter_parity build failed:\n{res.stderr}")
    return BIN
