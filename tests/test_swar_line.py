"""The parser's eight-bytes-at-a-time line decoder (kc_cuda_b200/csrc/swar_line.h),
compiled for the host, against the byte-at-a-time grammar of the reference parser
(src/kc_gpu.cpp:243-306): on every line it takes, it must give the same two numbers
(or a blank line); the lines it leaves to the byte loop are only checked to be few
among well-formed ones."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "kc_cuda_b200", "csrc")

HARNESS = r"""
#include <string.h>
#include "swar_line.h"
extern "C" int decode(const unsigned char* p, unsigned* x, unsigned* y, int* blank) {
  uint64_t w[3];
  memcpy(w, p, 24);
  bool b = false;
  const bool ok = kt::swar::decode_line(w, x, y, &b);
  *blank = b;
  return ok;
}
"""


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("swar")
    src = d / "h.cpp"
    so = d / "h.so"
    src.write_text(HARNESS)
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", HEADER_DIR, str(src), "-o", str(so)],
                   check=True)
    L = ctypes.CDLL(str(so))
    L.decode.restype = ctypes.c_int
    L.decode.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint),
                         ctypes.POINTER(ctypes.c_int)]
    return L


def grammar(line: bytes):
    """('blank',) / ('one', x) / ('two', x, y): the reference grammar on one line
    (bytes up to its newline); digits are bytes 0x30..0x7f adding byte - 0x30,
    values wrap at 2^32."""
    def digit(b):
        return 0x30 <= b <= 0x7F
    i, n = 0, len(line)
    while i < n and not digit(line[i]):
        i += 1
    if i == n:
        return ("blank",)
    x = 0
    while i < n and digit(line[i]):
        x = (x * 10 + line[i] - 0x30) & 0xFFFFFFFF
        i += 1
    while i < n and not digit(line[i]):
        i += 1
    if i == n:
        return ("one", x)
    y = 0
    while i < n and digit(line[i]):
        y = (y * 10 + line[i] - 0x30) & 0xFFFFFFFF
        i += 1
    return ("two", x, y)


def check(L, window: bytes):
    assert len(window) >= 24
    line = window.split(b"\n", 1)[0]
    x, y, blank = ctypes.c_uint(), ctypes.c_uint(), ctypes.c_int()
    ok = L.decode(window[:24], ctypes.byref(x), ctypes.byref(y), ctypes.byref(blank))
    if not ok:
        return False
    want = grammar(line)
    if blank.value:
        assert want == ("blank",), (window, want)
    else:
        assert want == ("two", x.value, y.value), (window, want, x.value, y.value)
    return True


def rand_line(rng) -> bytes:
    kind = rng.integers(0, 10)
    def num():
        return str(int(rng.integers(0, 10 ** int(rng.integers(1, 11))))).encode()
    seps = [b"\t", b" ", b"\t\t", b" \t", b",", b"\r\t"]
    odd = [b":", b"A", b"\x80", b"\xff", b"/", b"~", b"\x00", b"\r"]
    if kind <= 4:
        return num() + seps[int(rng.integers(0, len(seps)))] + num() + b"\n"
    if kind == 5:
        return b"\n" if rng.integers(0, 2) else b"  \t \n"
    if kind == 6:
        return num() + b"\n"
    if kind == 7:
        parts = [num(), odd[int(rng.integers(0, len(odd)))], num(), b"\t", num()]
        return b"".join(parts[: int(rng.integers(2, 6))]) + b"\n"
    if kind == 8:
        return odd[int(rng.integers(0, len(odd)))] + num() + b"\t" + num() + b"\t" + num() + b"\n"
    return b" " * int(rng.integers(0, 30)) + num() + b"\t" + num() + b"\r\n"


def test_swar_decoder_matches_grammar(lib):
    rng = np.random.default_rng(11)
    taken = 0
    for _ in range(20000):
        lines = b"".join(rand_line(rng) for _ in range(4))
        window = lines + b"\x00" * 24
        if check(lib, window):
            taken += 1
    assert taken > 5000


def test_swar_decoder_takes_well_formed_lines(lib):
    """Lines "x\\ty\\n" with ids below 10^8 all take the fast path."""
    rng = np.random.default_rng(12)
    for _ in range(5000):
        x, y = (int(v) for v in rng.integers(0, 10 ** 8, size=2))
        window = f"{x}\t{y}\n".encode() + f"{y}\t{x}\n".encode() + b"\x00" * 24
        assert check(lib, window), window


@pytest.mark.parametrize("window,want", [
    (b"12\t34\n" + b"9" * 30, ("two", 12, 34)),
    (b"\n" + b"5\t6\n" * 8, ("blank",)),
    (b"0\t0\n" + b"\x00" * 24, ("two", 0, 0)),
    (b"99999999\t12345678\nxx" + b"\x00" * 8, ("two", 99999999, 12345678)),
    (b"  7 8 9\n" + b"\x00" * 24, ("two", 7, 8)),
])
def test_swar_decoder_cases(lib, window, want):
    assert check(lib, window)
    assert grammar(window.split(b"\n", 1)[0]) == want


@pytest.mark.parametrize("window", [
    b"123456789\t1\n" + b"\x00" * 24,     # nine digits: the byte loop
    b"12:3\t4\n" + b"\x00" * 24,          # ':' is a digit of the grammar
    b"5\n6\t7\n" + b"\x00" * 24,          # one number on the line
    b" " * 24 + b"1\t2\n",                # no newline or digit in the window
])
def test_swar_decoder_leaves_the_rest(lib, window):
    x, y, blank = ctypes.c_uint(), ctypes.c_uint(), ctypes.c_int()
    assert not lib.decode(window[:24], ctypes.byref(x), ctypes.byref(y), ctypes.byref(blank))
