# SPDX-License-Identifier: MIT
"""The pm* driver library on the host (no GPU needed).

- libpm_b200_driver.so exports exactly the four loader entry points of the
  reference's driver ABI (include/parallel_mater/pm_driver.h:34-41) and
  resolves commands by name with the reference's null-handle rules
  (src/driver/slang/entry.cpp:30-56).
- Commands of domains the driver does not provide resolve to NULL, which
  the reference loader turns into PM_ERROR_FEATURE_NOT_PRESENT.
- Instance creation validates like src/api/instance.cpp:420-469.
- When the reference checkout is present, every struct, field offset and
  enumerator of include/pm_b200.h matches the reference header's.
"""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from pmb200 import pm

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
HEADER = os.path.join(REPO, "include", "pm_b200.h")
REF_INCLUDE = os.path.join(os.environ.get("PMB_REFERENCE_ROOT", "/root/reference"), "include")
ENTRY_POINTS = {"pm_driverNegotiateLoaderInterfaceVersion", "pm_driverGetInstanceProcAddr",
                "pm_driverGetDeviceProcAddr", "pm_driverGetPhysicalDeviceProcAddr"}


@pytest.fixture(scope="module")
def drv():
    if not os.path.exists(pm.DRIVER_PATH):
        pytest.skip("driver not built")
    return pm.driver()


def test_exports_exactly_the_driver_abi(drv):
    out = subprocess.run(["nm", "-D", "--defined-only", pm.DRIVER_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported == ENTRY_POINTS


def test_negotiate_interface_version(drv):
    v = ctypes.c_uint32(7)
    assert drv.pm_driverNegotiateLoaderInterfaceVersion(ctypes.byref(v)) == 0 and v.value == 2
    v = ctypes.c_uint32(1)
    assert drv.pm_driverNegotiateLoaderInterfaceVersion(ctypes.byref(v)) == 0 and v.value == 1
    v = ctypes.c_uint32(0)
    assert drv.pm_driverNegotiateLoaderInterfaceVersion(ctypes.byref(v)) == pm.ERROR_INVALID_ARGUMENT
    assert drv.pm_driverNegotiateLoaderInterfaceVersion(None) == pm.ERROR_INVALID_ARGUMENT


def test_proc_lookup_rules(drv):
    gi, gd, gp = drv.pm_driverGetInstanceProcAddr, drv.pm_driverGetDeviceProcAddr, \
        drv.pm_driverGetPhysicalDeviceProcAddr
    for name in (b"pmCreateInstance", b"pmEnumerateInstanceVersion", b"pmGetInstanceProcAddr"):
        assert gi(None, name), name
    for name in (b"pmCreateDevice", b"pmCmdStepSimulation", b"pmQueueSubmit"):
        assert not gi(None, name), name
        assert not gd(None, name), name
        assert not gp(None, name), name
    assert not gi(None, None)


def _instance():
    api = pm.Api()
    inst = ctypes.c_void_p()
    rc = api.pmCreateInstance(ctypes.byref(pm.InstanceCreateInfo(pm.ST_INSTANCE, None, pm.API_VERSION_0_3)),
                              None, ctypes.byref(inst))
    assert rc == pm.SUCCESS
    return inst


def test_every_rigid_command_resolves_and_other_domains_do_not(drv):
    inst = _instance()
    try:
        for name in pm.SIGNATURES:
            assert drv.pm_driverGetInstanceProcAddr(inst, name.encode()), name
        for name in ("pmCmdWriteFluidParticles", "pmCreateFluid", "pmCmdWriteCloth", "pmCmdCopyDebugData",
                     "pmImportNativeDevice", "pmCmdWriteSmoke", "pmNotACommand"):
            assert not drv.pm_driverGetInstanceProcAddr(inst, name.encode()), name
    finally:
        pm.Api(instance=inst).pmDestroyInstance(inst)


def test_instance_creation_validates(drv):
    api = pm.Api()
    inst = ctypes.c_void_p()
    bad = pm.InstanceCreateInfo(pm.ST_DEVICE, None, pm.API_VERSION_0_3)
    assert api.pmCreateInstance(ctypes.byref(bad), None, ctypes.byref(inst)) == pm.ERROR_INVALID_ARGUMENT
    old = pm.InstanceCreateInfo(pm.ST_INSTANCE, None, (0 << 22) | (2 << 12))
    assert api.pmCreateInstance(ctypes.byref(old), None, ctypes.byref(inst)) == pm.ERROR_INCOMPATIBLE_VERSION
    assert api.pmCreateInstance(None, None, ctypes.byref(inst)) == pm.ERROR_INVALID_ARGUMENT
    v = ctypes.c_uint32()
    assert api.pmEnumerateInstanceVersion(ctypes.byref(v)) == 0 and v.value == pm.API_VERSION_0_3


def test_physical_devices_match_cuda_devices(drv):
    inst = _instance()
    api = pm.Api(instance=inst)
    try:
        n = ctypes.c_uint32()
        assert api.pmEnumeratePhysicalDevices(inst, ctypes.byref(n), None) == 0
        try:
            import torch
            expected = torch.cuda.device_count() if torch.cuda.is_available() else 0
        except ImportError:
            expected = n.value
        assert n.value == expected
    finally:
        api.pmDestroyInstance(inst)


# ---------------------------------------------------------------- ABI layout
def _structs_and_enums():
    text = open(HEADER).read()
    structs = {}
    for m in re.finditer(r"typedef struct (Pm\w+) \{(.*?)\} \1;", text, re.S):
        fields = []
        for line in m.group(2).split(";"):
            line = line.strip()
            if not line:
                continue
            f = re.search(r"(\w+)\s*(\[[^\]]*\])*\s*$", line)
            fields.append(f.group(1))
        structs[m.group(1)] = fields
    enums = re.findall(r"^\s+(PM_[A-Z0-9_]+) = ", text, re.M)
    defines = [d for d, value in re.findall(r"^#define (PM_[A-Z0-9_]+) (.*)$", text, re.M)
               if not value.startswith('"') and d not in ("PM_MAKE_API_VERSION", "PM_B200_DRIVER_API")]
    return structs, enums, defines


def _layout_program(include_line, structs, enums, defines):
    lines = ["#include <stdio.h>", "#include <stddef.h>", include_line, "int main(void) {"]
    for s, fields in structs.items():
        lines.append(f'printf("{s} %zu %zu\\n", sizeof({s}), _Alignof({s}));')
        for f in fields:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    for e in enums + defines:
        lines.append(f'printf("{e} %llu\\n", (unsigned long long)({e}));')
    lines.append("return 0; }")
    return "\n".join(lines)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_INCLUDE, "parallel_mater", "parallel_mater.h")),
                    reason="reference checkout absent")
@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_abi_layout_matches_reference_header(tmp_path):
    structs, enums, defines = _structs_and_enums()
    assert len(structs) >= 45 and len(enums) >= 60
    outputs = []
    for tag, inc, flags in (("ours", f'#include "{HEADER}"', []),
                            ("ref", "#include <parallel_mater/parallel_mater.h>\n"
                                    "#include <parallel_mater/pm_driver.h>", ["-I", REF_INCLUDE])):
        src = tmp_path / f"{tag}.c"
        exe = tmp_path / tag
        src.write_text(_layout_program(inc, structs, enums, defines))
        subprocess.run(["gcc", "-std=c11", *flags, str(src), "-o", str(exe)], check=True)
        outputs.append(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    ours, ref = outputs
    assert ours == ref


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_INCLUDE, os.pardir, "tests", "api", "driver_abi_tests.cpp")),
                    reason="reference checkout absent")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_reference_driver_abi_test_passes_its_driver_checks(tmp_path):
    """The reference's own tests/api/driver_abi_tests.cpp, compiled unmodified
    against the reference headers and run on libpm_b200_driver.so: the four
    loader entry points resolve, no pm* command is exported, the interface
    version negotiates, instance-level lookups with a null instance answer
    pmCreateInstance but not device commands, and a newer API version is
    refused without creating an instance. Its second half opens the
    reference loader library, which needs the reference's generated
    registry sources to build; it is pointed at a path that does not exist,
    so the run must stop exactly at that check, after every driver check
    passed."""
    src = os.path.normpath(os.path.join(REF_INCLUDE, os.pardir, "tests", "api", "driver_abi_tests.cpp"))
    exe = tmp_path / "driver_abi_tests"
    subprocess.run(["g++", "-std=c++20", "-I", REF_INCLUDE, src, "-o", str(exe), "-ldl"], check=True)
    out = subprocess.run([str(exe), pm.DRIVER_PATH, str(tmp_path / "no_loader.so")], capture_output=True, text=True)
    assert out.returncode == 1
    failed = [line for line in out.stderr.splitlines() if line.startswith("line ")]
    assert len(failed) == 1 and failed[0].endswith("loader != nullptr"), out.stderr
