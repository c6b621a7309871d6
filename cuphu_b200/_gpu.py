"""GPU queries (reference cuphu/_gpu.py:6-18, cuphu_py.cu:435-456)."""
import ctypes as C

from cuphu_b200._lib import check, lib


def gpu_count() -> int:
    """Number of CUDA devices visible to this process."""
    return int(lib().cuphu_gpu_count())


def gpu_name(device_id: int = 0) -> str:
    buf = C.create_string_buffer(256)
    check(lib().cuphu_gpu_name(int(device_id), buf, 256))
    return buf.value.decode()


def gpu_info(device_id: int = 0) -> dict:
    """Device properties under the reference's keys (cuphu_py.cu:445-456):
    name, total_memory (bytes), sm_count and compute_cap ("major.minor")."""
    mem = C.c_longlong()
    sms, ma, mi = C.c_int(), C.c_int(), C.c_int()
    check(lib().cuphu_gpu_info(int(device_id), C.byref(mem), C.byref(sms), C.byref(ma),
                               C.byref(mi)))
    return {"name": gpu_name(device_id), "total_memory": int(mem.value),
            "sm_count": int(sms.value), "compute_cap": f"{int(ma.value)}.{int(mi.value)}"}
