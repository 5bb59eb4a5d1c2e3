"""Writes tests/golden/lda_full.bin and lda_model_only.bin with tomotopy's
own serializer (oracle/_ref/libtmtserial.so, compiled from the tomotopy
tree by oracle/Makefile) for a small, self-consistent LDA state, and the
fields into lda_fields.npz.  Run where the tomotopy tree exists:
    make -C oracle && python tests/golden/make_model_golden.py"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "..", "oracle", "_ref", "libtmtserial.so")


def main():
    lib = C.CDLL(LIB)
    V_ = C.c_void_p
    lib.ref_write_lda.argtypes = [C.c_char_p, C.c_uint32, V_, V_, C.c_uint64, C.c_uint64, V_, C.c_uint64, C.c_float,
                                  V_, C.c_float, C.c_uint16, C.c_uint32, C.c_uint32, V_, V_, C.c_int, C.c_uint64,
                                  V_, V_, V_, V_, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_uint64)]
    lib.ref_free.argtypes = [C.POINTER(C.c_uint8)]
    rng = np.random.default_rng(20261203)
    K, nv = 7, 40
    vocab = [f"w{i}" for i in range(nv - 3)] + ["été", "naïve", "x"]
    realV = nv - 4                       # the last 4 ids are removed words
    D = 12
    lens = rng.integers(0, 25, D)
    lens[3] = 0
    doc_off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    words = np.concatenate([np.sort(rng.integers(0, nv, n)) for n in lens]).astype(np.uint32)
    w_order = np.concatenate([rng.permutation(n) for n in lens]).astype(np.uint32)
    zs = rng.integers(0, K, len(words)).astype(np.uint16)
    zs[words >= realV] = 0xFFFF
    nkw = np.zeros((realV, K), np.int32)
    nk = np.zeros(K, np.int32)
    for w, z in zip(words, zs):
        if w < realV:
            nkw[w, z] += 1
            nk[z] += 1
    cf = np.bincount(words, minlength=nv).astype(np.uint64)
    df = np.zeros(nv, np.uint64)
    for d in range(D):
        df[np.unique(words[doc_off[d]:doc_off[d + 1]])] += 1
    alphas = (0.05 * (1 + np.arange(K))).astype(np.float32)
    extra = bytes(range(37))
    vb = ("\0".join(vocab) + "\0").encode("utf-8")
    eb = np.frombuffer(extra, np.uint8).copy()
    for full, name in ((1, "lda_full.bin"), (0, "lda_model_only.bin")):
        out = C.POINTER(C.c_uint8)()
        n = C.c_uint64()
        lib.ref_write_lda(vb, nv, cf.ctypes.data_as(V_), df.ctypes.data_as(V_), realV, 123, eb.ctypes.data_as(V_),
                          len(eb), float(alphas[0]), alphas.ctypes.data_as(V_), 0.02, K, 5, 10,
                          nk.ctypes.data_as(V_), nkw.ctypes.data_as(V_), full, D, doc_off.ctypes.data_as(V_),
                          words.ctypes.data_as(V_), w_order.ctypes.data_as(V_), zs.ctypes.data_as(V_),
                          C.byref(out), C.byref(n))
        data = C.string_at(out, n.value)
        lib.ref_free(out)
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)
    np.savez_compressed(os.path.join(HERE, "lda_fields.npz"), K=K, nv=nv, realV=realV, doc_off=doc_off, words=words,
                        w_order=w_order, zs=zs, nkw=nkw, nk=nk, cf=cf, df=df, alphas=alphas,
                        vocab=np.array(vocab), extra=eb)
    print("wrote golden model files")


if __name__ == "__main__":
    main()
