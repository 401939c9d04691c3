"""B200-native path-tracing hot path for flarive/CortexRaytracerCuda's render call.

Layout:
  csrc/         sm_100a kernels (render_compat.cu, render_clean.cu) and the host C ABI (rtc_api.cpp,
                bvh_build.cpp) built into librtc_b200.so by build.py
  scene.py      scene description (mirror of include/rtc.h)
  configs.py    synthetic scenes of the measured workloads
  renderer.py   Context / DeviceScene / GpuB200Renderer / launch_gpu over the C ABI
"""
from .scene import (BG_CONSTANT, BG_ENV_MAP, BG_SKY_GRADIENT, DRAW_ORDER_DEVICE, DRAW_ORDER_HOST, MODE_CLEAN,
                    MODE_COMPAT, Camera, RenderParams, Scene)

__all__ = ["Scene", "Camera", "RenderParams", "MODE_COMPAT", "MODE_CLEAN", "DRAW_ORDER_DEVICE", "DRAW_ORDER_HOST",
           "BG_CONSTANT", "BG_SKY_GRADIENT", "BG_ENV_MAP"]
