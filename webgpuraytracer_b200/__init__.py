"""B200-native progressive path tracer: a drop-in for the WebGPU renderer of
DragonFireGames/WebGPURaytracer (shader.wgsl, denoiser.wgsl, scale.wgsl behind tracer.js's
Renderer/Denoiser), as CUDA kernels for sm_100a behind a C ABI (include/wgpt.h).

    from webgpuraytracer_b200 import synth, renderer
    s = synth.small_scene()
    r = renderer.Renderer(256, 256)
    r.set_scene(s)
    r.render(tsize=256, reps=16)
    img = r.read_output()
"""
__all__ = ["scene", "renderer", "synth", "glmat", "build"]
