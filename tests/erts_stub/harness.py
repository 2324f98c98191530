"""Loads nif/nx_stereo_cuda_nif.cpp built against the fake runtime in this
directory (TEST INFRASTRUCTURE ONLY) and calls its functions as the BEAM
would: terms are the fake's handles, messages come back printed."""
import ctypes
import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BUILD = os.path.join(HERE, "_build")
LIBRARY = os.path.join(BUILD, "nif_under_fake_erts.so")


class Func(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("arity", ctypes.c_uint),
                ("fptr", ctypes.c_void_p), ("flags", ctypes.c_uint)]


class Entry(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("num_of_funcs", ctypes.c_int),
                ("funcs", ctypes.POINTER(Func)), ("load", ctypes.c_void_p)]


def build():
    from nx_stereo_b200 import build as library

    library.build()
    sources = [os.path.join(ROOT, "nif", "nx_stereo_cuda_nif.cpp"), os.path.join(HERE, "fake_erts.cpp"),
               os.path.join(HERE, "erl_nif.h"),
               os.path.join(ROOT, "nx_stereo_b200", "csrc", "port_records.h")]
    if os.path.exists(LIBRARY) and os.path.getmtime(LIBRARY) >= max(map(os.path.getmtime, sources)):
        return LIBRARY
    os.makedirs(BUILD, exist_ok=True)
    lib_dir = os.path.join(ROOT, "nx_stereo_b200")
    subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-I", HERE, "-o", LIBRARY + ".tmp",
                    sources[0], sources[1], "-L", lib_dir, "-lnxs_b200", f"-Wl,-rpath,{lib_dir}",
                    "-lpthread"], check=True)
    os.replace(LIBRARY + ".tmp", LIBRARY)
    return LIBRARY


class Nif:
    def __init__(self):
        self.lib = ctypes.CDLL(build())
        T = ctypes.c_size_t
        for name, res, args in [("fake_int", T, [ctypes.c_longlong]), ("fake_pid", T, [ctypes.c_longlong]),
                                ("fake_ref", T, [ctypes.c_longlong]),
                                ("fake_binary", T, [ctypes.c_char_p, ctypes.c_size_t]),
                                ("fake_print", ctypes.c_int, [T, ctypes.c_char_p, ctypes.c_int]),
                                ("fake_next_message", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
                                ("fake_process_down", None, [ctypes.c_longlong]),
                                ("fake_env", ctypes.c_void_p, [])]:
            fn = getattr(self.lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib.nif_init.restype = ctypes.POINTER(Entry)
        entry = self.lib.nif_init().contents
        self.module = entry.name.decode()
        load = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, T)(entry.load)
        assert load(self.lib.fake_env(), None, 0) == 0
        self.funcs = {}
        for i in range(entry.num_of_funcs):
            f = entry.funcs[i]
            proto = ctypes.CFUNCTYPE(T, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(T))
            self.funcs[(f.name.decode(), f.arity)] = (proto(f.fptr), f.flags)

    def call(self, name, *args):
        fn, _ = self.funcs[(name, len(args))]
        argv = (ctypes.c_size_t * len(args))(*args)
        return fn(self.lib.fake_env(), len(args), argv)

    def text(self, term):
        buf = ctypes.create_string_buffer(1 << 22)
        self.lib.fake_print(term, buf, len(buf))
        return buf.value.decode()

    def binary(self, data):
        return self.lib.fake_binary(data, len(data))

    def message(self, timeout=30.0):
        buf = ctypes.create_string_buffer(1 << 24)
        deadline = time.monotonic() + timeout
        while time.monotonic() < deadline:
            if self.lib.fake_next_message(buf, len(buf)):
                return buf.value.decode()
            time.sleep(0.002)
        return None


def hex_binary(text):
    """The bytes of a printed binary <<...>>."""
    return bytes.fromhex(text[2:-2])
