"""The drop-in boundary, driven by the reference's own code generator (CPU).

tests/golden/visitor/*.sycl are the programs JITOperatorVisitor::generateCode
(src/core/visitor.cpp:4771-4878) emits for the measured query shapes.  Handed
to cx_compile unchanged -- as the reference's ICompiler::compile would hand it
the visitor's text -- each is translated to this library's launch skeleton,
compiled by NVRTC for sm_100a (no device needed) and carries the result shape
the visitor chose.  Where the reference sources are mounted, the fixtures are
checked to be exactly what its generator emits today, and the adapters of the
reference's ICompiler / IExecutor interfaces compile against its own
include/core/execution.h."""
import os
import subprocess
from pathlib import Path

import pytest

from practice_b200 import _lib

from visitor_plans import TRANSLATED, plan

ROOT = Path(__file__).resolve().parent.parent
FIX = ROOT / "tests" / "golden" / "visitor"
REF = Path(os.environ.get("CRYSTAL_REFERENCE", "/root/reference"))


@pytest.mark.parametrize("name", TRANSLATED)
def test_visitor_program_compiles_through_cx_compile(name):
    src = (FIX / f"{name}.sycl").read_text()
    assert 'extern "C" void execute_query(db::ExecutionContext* ctx)' in src and "sycl::" in src
    t = _lib.translate_visitor(src)
    assert "sycl::" not in t and "__global__" in t and t.startswith("/*@cx-launch")
    m = _lib.Module(src, key=f"visitor_{name}")  # the untranslated text goes straight to cx_compile
    p = plan(name, 1000)
    assert m.info.result_words == p.group_slots * p.storage_ts
    assert m.info.storage_ts == p.storage_ts
    # Every primitive call of the visitor's kernels survives the translation.
    for call in ("BlockLoad<int, BLOCK_THREADS, ITEMS_PER_THREAD>", "InitFlags<BLOCK_THREADS, ITEMS_PER_THREAD>"):
        assert src.count(call) == t.count(call)
    if name != "t0":
        assert t.count("BlockProbeAndPHT_") == src.count("BlockProbeAndPHT_") > 0
    if any(f"*{m}" in src for m in ("C_LEN", "S_LEN", "P_LEN")):
        assert "htrows" in t  # C_LEN / S_LEN / P_LEN tables are sized by the context's rows


def test_dense_materialisation_is_refused_with_its_reason():
    src = (FIX / "q31_nullable.sycl").read_text()
    with pytest.raises(_lib.CxError) as e:
        _lib.translate_visitor(src)
    assert "dense result materialisation" in str(e.value) or "host-side block" in str(e.value)


def test_foreign_or_broken_programs_are_refused():
    src = (FIX / "q31.sycl").read_text()
    with pytest.raises(_lib.CxError):
        _lib.translate_visitor(src.replace("C_LEN", "X_LEN"))
    with pytest.raises(_lib.CxError):
        _lib.translate_visitor(src.replace("sycl::nd_item<1> it", "sycl::item<1> it"))
    with pytest.raises(_lib.CxError):
        _lib.Module("int main() { return 0; }", key="not_a_program")


@pytest.mark.skipif(not (REF / "src" / "core" / "visitor.cpp").exists(), reason="reference sources not mounted")
@pytest.mark.parametrize("name", TRANSLATED + ["q31_nullable"])
def test_fixtures_are_what_the_reference_generator_emits(name):
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "visitor", f"REF={REF}"], check=True, capture_output=True)
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "emit_visitor"), name], check=True, capture_output=True,
                         text=True).stdout
    assert out == (FIX / f"{name}.sycl").read_text()


@pytest.mark.skipif(not (REF / "include" / "core" / "execution.h").exists(), reason="reference sources not mounted")
def test_adapters_compile_against_the_reference_interfaces(tmp_path):
    """NvrtcCompiler / CudaModuleExecutor compile against the reference's own
    include/core/execution.h (ICompiler, IExecutor, ExecutionContext) with a
    declaration-only SYCL header; every member they touch exists there."""
    unit = tmp_path / "adapters.cpp"
    unit.write_text('#include "execution_b200.h"\n'
                    'static_assert(!std::is_abstract_v<db::NvrtcCompiler>);\n'
                    'static_assert(!std::is_abstract_v<db::CudaModuleExecutor>);\n'
                    'std::unique_ptr<db::ICompiler> make_c() { return std::make_unique<db::NvrtcCompiler>(); }\n'
                    'std::unique_ptr<db::IExecutor> make_e(std::shared_ptr<Catalog> c) {\n'
                    '  return std::make_unique<db::CudaModuleExecutor>(c); }\n')
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-include", "type_traits", f"-I{ROOT / 'tests' / 'shims'}",
           f"-I{REF / 'include'}", f"-I{ROOT / 'include'}", f"-I{ROOT / 'practice_b200' / 'adapters'}", str(unit)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]
