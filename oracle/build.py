"""ORACLE -- test infrastructure only. Builds the oracle libraries.

* oracle/_build/libkmeans_oracle.so from oracle/kmeans_oracle.c,
  oracle/kmeans_csr_oracle.c and oracle/kmeans_init_oracle.cpp (always);
* oracle/_ref/libkmeans_daal_ref.so from the reference tree via
  oracle/ref/Makefile, when that tree is present (it is absent on GPU hosts,
  which use the prebuilt library that travels with the working tree).
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_LIB = os.path.join(HERE, "_build", "libkmeans_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libkmeans_daal_ref.so")
# The reference source tree this recipe compiles from: ONEDAL_REFERENCE_TREE, or
# where this build environment mounts it. The only place the path is named.
REFERENCE_TREE = os.environ.get("ONEDAL_REFERENCE_TREE", "/root/reference")


def build_restated(force: bool = False) -> str:
    src = os.path.join(HERE, "kmeans_oracle.c")
    src_csr = os.path.join(HERE, "kmeans_csr_oracle.c")
    src_init = os.path.join(HERE, "kmeans_init_oracle.cpp")
    newest = max(os.path.getmtime(src), os.path.getmtime(src_csr), os.path.getmtime(src_init))
    if force or not os.path.exists(RESTATED_LIB) or os.path.getmtime(RESTATED_LIB) < newest:
        out = os.path.dirname(RESTATED_LIB)
        os.makedirs(out, exist_ok=True)
        obj_c, obj_cpp = os.path.join(out, "kmeans_oracle.o"), os.path.join(out, "kmeans_init_oracle.o")
        obj_csr = os.path.join(out, "kmeans_csr_oracle.o")
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-std=c11", "-c", "-o", obj_c, src])
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-std=c11", "-c", "-o", obj_csr, src_csr])
        # strict IEEE arithmetic; the FMA the restatement needs is written explicitly
        subprocess.check_call(["g++", "-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-c", "-o", obj_cpp,
                               src_init])
        subprocess.check_call(["g++", "-fopenmp", "-shared", "-o", RESTATED_LIB, obj_c, obj_csr, obj_cpp])
    return RESTATED_LIB


def build_reference() -> str | None:
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "cpp", "daal")):
        return REF_LIB if os.path.exists(REF_LIB) else None
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={REFERENCE_TREE}",
                           f"-j{os.cpu_count() or 4}"])
    return REF_LIB


def build_all() -> None:
    build_restated()
    build_reference()


if __name__ == "__main__":
    build_all()
