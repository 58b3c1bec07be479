"""Frame configurations (the fields of ap_frame_config, include/appearance_cuda.h).

`faithful` is the reference's PathTracerGpuConfig::default() with the pass
literals hard-coded in crates/appearance-path-tracer-gpu/src/lib.rs:220-245,413-545
and the shader constants (NUM_AREA_SAMPLES 4, helpers/nee.wgsl:125; DI spatial
NUM_SAMPLES 3, restir_di_spatial.wgsl:15; GI spatial 5, restir_gi_spatial.wgsl:16;
M caps restir_di_temporal.wgsl:159, restir_gi_temporal.wgsl:100).
"""

FAITHFUL = dict(
    max_bounces=2, sample_count=1, restir_di=1, restir_gi=1, svgf=0, firefly_filter=1, taa=0,
    di_area_samples=4, di_bsdf_samples=1, di_temporal_m_factor=20.0,
    di_spatial_passes=1, di_spatial_samples=3, di_unbiased=1,
    gi_temporal_m_cap=30.0, gi_spatial_passes=0, gi_spatial_samples=5, gi_unbiased=1,
    svgf_max_history=24, svgf_atrous_passes=5, taa_history_influence=0.8)

# Cornell box, 512x512, 16 spp, depth 5, no reuse or denoising: the plain
# estimator of the frame (RIS next-event estimation + resampled continuation).
PLAIN = dict(FAITHFUL, max_bounces=5, sample_count=16, restir_di=0, restir_gi=0, firefly_filter=0)

# 1920x1080 real-time frame: depth 8, 1 spp, ReSTIR DI with 32 area candidates,
# temporal reuse (M cap 20x) and 5-neighbour spatial reuse, ReSTIR GI with
# temporal reuse (spatial GI reuse off, as the reference runs it,
# crates/appearance-path-tracer-gpu/src/lib.rs:441), firefly filter, SVGF with 5
# a-trous passes, TAA.
REALTIME = dict(FAITHFUL, max_bounces=8, sample_count=1, svgf=1, taa=1, di_area_samples=32,
                di_spatial_samples=5)

# REALTIME plus one unbiased 5-neighbour ReSTIR GI spatial pass.
REALTIME_GI_SPATIAL = dict(REALTIME, gi_spatial_passes=1, gi_spatial_samples=5)

PRESETS = dict(faithful=FAITHFUL, plain=PLAIN, realtime=REALTIME, realtime_gi_spatial=REALTIME_GI_SPATIAL)
