"""Builds tests/cpp/api_client.cpp against the library (g++, the C++ API
headers under include/) for the C++-host tests."""
import os
import subprocess

import unblending_b200 as U

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(tmpdir) -> str:
    exe = os.path.join(str(tmpdir), "api_client")
    libdir = os.path.dirname(U.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "api_client.cpp"), "-o", exe, U.LIB_PATH,
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    return exe
