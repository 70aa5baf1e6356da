/*
 * gjxl_b200 — C ABI of the B200 (sm_100a) perceptual-analysis backend for the
 * gjxl JPEG XL VarDCT encoder.
 *
 * Conventions
 *  - All image pointers are DEVICE pointers unless a name says "host".
 *  - A three-plane image is one base pointer: plane c starts at
 *    base + c * plane_pitch elements; rows are `stride` elements apart.
 *    Strides and plane pitches are multiples of 4 elements and bases are
 *    16-byte aligned (the kernels use 128-bit accesses).
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy stream).
 *  - Return values are the reference's StatusCode numbering
 *    (src/core/status.h:12-22): 0 ok, 1 invalid argument, 2 unsupported,
 *    3 unavailable, 4 out of memory, 5 failed precondition,
 *    6 submission failed, 7 device error, 8 internal.
 *    gjxl_b200_last_error() returns the thread's last message.
 *  - `device_error` (may be NULL) is a device uint32 word the kernels OR
 *    bits into: 1 non-finite input, 2 non-finite output, 4 range, 8 internal.
 *    Callers map a nonzero word to StatusCode 7 (the reference's
 *    ReadAndCheckDeviceError, src/gpu/cuda/cuda_aq_resident.cpp:3451).
 */
#ifndef GJXL_B200_H_
#define GJXL_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GJXL_B200_API __attribute__((visibility("default")))
#else
#define GJXL_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GJXL_B200_OK 0
#define GJXL_B200_INVALID_ARGUMENT 1
#define GJXL_B200_UNSUPPORTED 2
#define GJXL_B200_UNAVAILABLE 3
#define GJXL_B200_OUT_OF_MEMORY 4
#define GJXL_B200_FAILED_PRECONDITION 5
#define GJXL_B200_SUBMISSION_FAILED 6
#define GJXL_B200_DEVICE_ERROR 7
#define GJXL_B200_INTERNAL 8

/* Thread-local description of the last failure (empty after success). */
GJXL_B200_API const char* gjxl_b200_last_error(void);

/* Library version (major * 10000 + minor * 100 + patch). */
GJXL_B200_API int gjxl_b200_version(void);

/*
 * Input preparation (row a1).
 * Replaces GpuResidentInputPreparation::PrepareResidentInput
 * (src/gpu/ops/resident_input.h:75-80) as implemented by
 * CudaBackend::PrepareResidentInput (src/gpu/cuda/cuda_input_preparation.cpp:299)
 * and LinearRgbToOpsinKernel (src/gpu/cuda/cuda_aq_exact_kernels.cu:45), fused
 * with the C API's packed sRGB decode (src/c_api/image_conversion.cpp:18-31,
 * 116-138).
 *
 * Reads packed 8-bit sRGB (channels = 3 RGB or 4 opaque RGBA; alpha ignored)
 * and writes the unpadded linear RGB planes (width x height) and the padded
 * XYB planes (padded_width x padded_height, padded by edge replication exactly
 * like color_transform_internal::LinearRgbToPaddedOpsin,
 * src/codec/color_transform.cpp:365).
 */
GJXL_B200_API int gjxl_b200_prepare_input(const uint8_t* pixels, size_t width, size_t height,
                            size_t row_stride_bytes, int channels,
                            float intensity_target, float* linear,
                            size_t linear_stride, size_t linear_plane_pitch,
                            float* opsin, size_t opsin_stride,
                            size_t opsin_plane_pitch, size_t padded_width,
                            size_t padded_height, uint32_t* device_error,
                            void* stream);

/*
 * Quantization-matrix scale statistics (row a2).
 * Replaces OpsinMatrixScaleStatsKernel (src/gpu/cuda/cuda_aq_exact_kernels.cu:100)
 * and ComputeQuantizationMatrixScaleStatsFromFiniteOpsin
 * (src/codestream/workflow.cpp:1318). Writes {x_edge, b_edge, exposed_blue}
 * as three device floats over the unpadded width x height region.
 * `stats` is cleared by this call.
 */
GJXL_B200_API int gjxl_b200_matrix_scale_stats(const float* opsin, size_t opsin_stride,
                                 size_t opsin_plane_pitch, size_t width,
                                 size_t height, float* stats, void* stream);

/*
 * Initial quantization field (row a3).
 * Replaces ComputeInitialQuantField (src/codec/adaptive_quantization.cpp:582)
 * as run on the GPU by InitialGradientKernel / FuzzyErosionKernel /
 * ModulationKernel (src/gpu/cuda/cuda_aq_kernels.cu:52,174,254) behind
 * PreparedAqEvaluation::ComputeInitialQuantization
 * (src/gpu/ops/aq_evaluation.h:219-396).
 *
 * Input: padded XYB (pre-Gaborish). Outputs: quant_field and strategy_mask,
 * one float per 8x8 block (dense, (padded_width/8) x (padded_height/8)), and
 * the blurred pixel mask (padded_width x padded_height, row stride
 * pixel_mask_stride). `scratch` is caller-provided device memory of at least
 * gjxl_b200_initial_quant_scratch_bytes() bytes, 16-byte aligned.
 */
GJXL_B200_API size_t gjxl_b200_initial_quant_scratch_bytes(size_t padded_width,
                                                           size_t padded_height);
GJXL_B200_API int gjxl_b200_initial_quant_field(
    const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
    size_t padded_width, size_t padded_height, float butteraugli_target,
    float rescale, float* quant_field, float* strategy_mask, float* pixel_mask,
    size_t pixel_mask_stride, void* scratch, size_t scratch_bytes,
    uint32_t* device_error, void* stream);

/*
 * Initial quantization field without any device allocation: no counterpart
 * in the reference. Same arguments and results as
 * gjxl_b200_initial_quant_field, but the scratch is a 16 MiB static device
 * array owned by the library, so the call allocates nothing. For callers that
 * cannot allocate device memory per image (a service under a fixed memory
 * budget, where cudaMalloc/cudaFree would synchronize the device and an
 * out-of-memory failure mid-image cannot be recovered; a plug-in host without
 * a device allocator).
 *  - Limit: padded images of at most 3,947,580 pixels (e.g. 2048 x 1920);
 *    larger ones are rejected with GJXL_B200_INVALID_ARGUMENT.
 *  - The first call on each device sets up the scratch address there
 *    (cudaGetSymbolAddress); make it before any stream capture.
 *  - One scratch array per device: overlapping calls on one device race.
 *    Serialize them (for example, on one stream).
 */
GJXL_B200_API int gjxl_b200_initial_quant_field_noalloc(
    const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
    size_t padded_width, size_t padded_height, float butteraugli_target,
    float rescale, float* quant_field, float* strategy_mask, float* pixel_mask,
    size_t pixel_mask_stride, uint32_t* device_error, void* stream);

/*
 * Inverse Gaborish (row a4).
 * Replaces GaborishInverseProvider::Apply
 * (src/codec/quantization_pipeline_internal.h:20-32) and GpuImagePrimitives'
 * Symmetric5 convolution (src/gpu/ops/primitives.h:68-85,
 * src/gpu/cuda/cuda_kernels.cu:1326). Three planes, mirrored borders, per-plane
 * multipliers (the reference's ApplyGaborishInverse, src/codec/gaborish.cpp:37).
 * `multipliers` is a HOST array of 3 floats. Input and output must not alias.
 */
GJXL_B200_API int gjxl_b200_gaborish_inverse(
    const float* input, size_t input_stride, size_t input_plane_pitch,
    float* output, size_t output_stride, size_t output_plane_pitch,
    size_t width, size_t height, const float* multipliers,
    uint32_t* device_error, void* stream);

/*
 * Initial chroma-from-luma map (row a5).
 * Replaces the CPU path's ComputeInitialColorCorrelationMap
 * (src/codec/chroma_from_luma.cpp:434) and the CUDA InitialCflKernel
 * (src/gpu/cuda/cuda_aq_kernels.cu:426) behind
 * PreparedQuantizationPipeline preprocessing
 * (src/codec/quantization_pipeline.cpp:155-213). Input: the Gaborish-inverted
 * padded XYB image. Outputs: int8 y_to_x and y_to_b per 64x64 tile (dense,
 * ceil(padded_width/64) x ceil(padded_height/64)). `opsin` 8-byte aligned,
 * stride and plane pitch even (floats).
 */
GJXL_B200_API int gjxl_b200_initial_cfl(const float* opsin, size_t opsin_stride,
                                        size_t opsin_plane_pitch,
                                        size_t padded_width,
                                        size_t padded_height, int8_t* y_to_x,
                                        int8_t* y_to_b, void* stream);

/*
 * The learned proposal network (row N4; no reference counterpart): 4
 * convolutions of 32 channels (3x3, BF16 with FP32 accumulation) over a
 * 64x64 tile of Gaborish-inverted XYB with an 8-px halo and log2 distance,
 * and a 1x1 head of 27 strategy logits and a log field scale per 8x8 block.
 * Parameters: gjxl_b200_cnn_param_count() FP32 values. The workspace holds
 * one batch of `tiles` inputs, activations and head outputs ([tiles][64][28]
 * FP32, copied to head_out when given). Training: one step computes the loss
 * (mean over all tiles * 64 block slots of weight * (softmax cross-entropy
 * against the label strategy + qf_weight * squared error of the log field
 * scale)) and the parameter gradients; AdamW updates the parameters.
 */
GJXL_B200_API size_t gjxl_b200_cnn_param_count(void);
GJXL_B200_API size_t gjxl_b200_cnn_workspace_bytes(int tiles);
GJXL_B200_API size_t gjxl_b200_cnn_train_scratch_bytes(int tiles);
GJXL_B200_API int gjxl_b200_cnn_gather(const float* opsin, size_t opsin_stride,
                                       size_t opsin_plane_pitch, size_t padded_width,
                                       size_t padded_height, const int* tile_list, int tiles,
                                       float distance, void* workspace, void* stream);
/* tensor_cores != 0: the convolutions as tcgen05 implicit GEMMs (what the
 * learned analysis runs); 0: the SIMT kernels the training step pairs with. */
GJXL_B200_API int gjxl_b200_cnn_forward(const float* params, int tiles, void* workspace,
                                        float* head_out, int tensor_cores, void* stream);
GJXL_B200_API int gjxl_b200_cnn_train_step(const float* params, int tiles, void* workspace,
                                           const uint8_t* labels, const float* targets,
                                           const float* weights, float qf_weight,
                                           float* grads, void* scratch, float* loss,
                                           void* stream);
GJXL_B200_API int gjxl_b200_cnn_adamw(float* params, const float* grads, float* m, float* v,
                                      int step, float lr, float beta1, float beta2, float eps,
                                      float weight_decay, void* stream);

/*
 * DC-group token streams (row f1): the DC residual and AC-metadata tokens of
 * every 256x256-block DC group, and their entropy-model histogram.
 * Replaces the CPU path's TokenizeSimpleDcGroupsForEncoder
 * (src/codestream/vardct/dc_group.cpp:469-546) with TokenizeWeightedDcGroup
 * (prediction 1, weighted_dc.cpp:47) or TokenizeSimpleDcGroup (prediction
 * 0, dc_group.cpp:291), and TokenizeSimpleAcMetadata (dc_group.cpp:349), as
 * called by the encoder at src/codestream/vardct/encoder.cpp:1930.
 * Inputs (device): quantized DC, 3 planes (X, Y, B) of blocks_x x blocks_y
 * int32 dc_plane_pitch elements apart; strategy cells ((strategy << 1) |
 * anchor); raw quant field; EPF sharpness (NULL: the default 4 everywhere);
 * y_to_x / y_to_b per 64x64 tile (ceil(blocks/8) per side).
 * Outputs (device): tokens as (context, value) uint32 pairs, EntropyToken's
 * layout, in the encoder's legacy context numbering (before the DC tree
 * layout's context map): dc_tokens (3 * blocks pairs; groups in row-major
 * order, channels Y, X, B, raster order), meta_tokens (per group: y_to_x
 * map, y_to_b map, anchor strategies, anchor quant fields, sharpness),
 * group_info (per group {dc_offset, dc_count, meta_offset, meta_count,
 * anchor_count}, in pairs), and optionally histogram: [45][128] uint32
 * counts of (context, hybrid-uint {4,2,0} symbol) over both streams.
 * Sizes from gjxl_b200_dc_token_sizes. A residual outside int32 or a quant /
 * sharpness / strategy the reference rejects sets device_error bit 2.
 */
GJXL_B200_API int gjxl_b200_dc_token_sizes(size_t blocks_x, size_t blocks_y,
                                           size_t* dc_tokens, size_t* meta_tokens,
                                           size_t* groups, size_t* scratch_bytes);
GJXL_B200_API int gjxl_b200_dc_tokenize(
    const int32_t* quantized_dc, size_t dc_plane_pitch, const uint8_t* cells,
    const int32_t* raw_quant, const uint8_t* epf_sharpness, const int8_t* y_to_x,
    const int8_t* y_to_b, size_t blocks_x, size_t blocks_y, int prediction,
    uint32_t* dc_tokens, uint32_t* meta_tokens, uint32_t* group_info, uint32_t* histogram,
    void* scratch, size_t scratch_bytes, uint32_t* device_error, void* stream);

/*
 * Default AC quantization matrix of one searched strategy and channel, in the
 * reference's coefficient layout (GetDefaultQuantizationMatrix,
 * src/codec/quantization.cpp:646-703). HOST outputs of `capacity` floats.
 */
GJXL_B200_API int gjxl_b200_quant_matrix(int strategy, int channel,
                                         float* dequant,
                                         float* inverse_dequant,
                                         size_t capacity);

/*
 * Precision of the AC-strategy candidate costs.
 *  EXACT: the reference CPU transform restated in FP64 (bit-identical costs,
 *         hence strategy grids, to the reference's CPU path).
 *  FAST:  the families with 16- or 32-pixel sides (DCT16x16, DCT32x16,
 *         DCT16x32, DCT32x32) as tcgen05 tensor-core MMAs on three-piece
 *         split-bf16 operands with f32 accumulation (FP32-class products),
 *         like the reference's own FP32 CUDA evaluator
 *         (src/gpu/cuda/cuda_kernels.cu:653); the 8-pixel families (DCT8,
 *         DCT16x8, DCT8x16) with FP32 fused multiply-adds on SIMT cores.
 *         Grids then match the exact mode except where a candidate's cost is
 *         within rounding of a tie.
 */
#define GJXL_B200_PRECISION_EXACT 0
#define GJXL_B200_PRECISION_FAST 1

/*
 * AC-strategy candidate costs (rows a6, a8).
 * Replaces GpuAcStrategyEvaluation (src/gpu/ops/ac_strategy.h:118-170) as run
 * by LaunchCudaAcStrategyBatch / FusedAcStrategyKernel
 * (src/gpu/cuda/cuda_ac_strategy.cpp:500-515, src/gpu/cuda/cuda_kernels.cu:653)
 * and the CPU EstimateAcStrategyCost (src/codec/ac_strategy.cpp:823).
 *
 * `opsin` is the Gaborish-inverted padded XYB image, `quant_field` the initial
 * field (dense blocks), `pixel_mask` the blurred mask, `y_to_x`/`y_to_b` the
 * initial CfL maps (dense 64x64 tiles). `costs` receives
 * gjxl_b200_ac_strategy_cost_bytes() bytes: seven planes (DCT8, DCT16x8,
 * DCT8x16, DCT16x16, DCT32x16, DCT16x32, DCT32x32) of one float per block,
 * valid at candidate anchors and NaN elsewhere.
 */
GJXL_B200_API size_t gjxl_b200_ac_strategy_cost_bytes(size_t padded_width,
                                                      size_t padded_height);
GJXL_B200_API int gjxl_b200_ac_strategy_costs(
    const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
    size_t padded_width, size_t padded_height, const float* quant_field,
    const float* pixel_mask, size_t pixel_mask_stride, const int8_t* y_to_x,
    const int8_t* y_to_b, float butteraugli_target, int dense_dct32,
    int precision, float* costs, uint32_t* device_error, void* stream);

/*
 * Candidate-batch evaluation (the reference's GpuAcStrategyEvaluation seam,
 * src/gpu/ops/ac_strategy.h:72-170): costs of `candidate_count` candidates of
 * one searched strategy, each an AcStrategyCandidate descriptor (24 bytes:
 * uint32 block_x, block_y; float quant_norm, entropy_multiplier, cfl_x,
 * cfl_b; device memory) into `costs` (device, one float per candidate).
 * `matrices`: the strategy's dequant X/Y/B then inverse dequant X/Y/B
 * (device; NULL: the default tables). With `quant_field` (and both CfL maps)
 * the quant norm and CfL factors are the device's own from the field, as in
 * the reference's resident form; otherwise the descriptors'. A descriptor
 * whose footprint leaves the image gets a NaN cost.
 */
GJXL_B200_API int gjxl_b200_ac_strategy_candidate_costs(
    int strategy, const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
    const float* pixel_mask, size_t pixel_mask_stride, size_t padded_width,
    size_t padded_height, const void* candidates, size_t candidate_count,
    const float* matrices, const float* quant_field, const int8_t* y_to_x,
    const int8_t* y_to_b, float butteraugli_target, int precision, float* costs,
    uint32_t* device_error, void* stream);
/*
 * AC-strategy search (rows a6, a7, a8): candidate costs followed by the
 * greedy hierarchical merge of every 64x64 tile on the device.
 * Replaces AcStrategySearchProvider::Find (src/codec/quantization_pipeline.h:34-50)
 * as implemented by FindAcStrategyGridGpuResident
 * (src/gpu/ops/ac_strategy_search.h:130) and FindAcStrategyGrid
 * (src/codec/ac_strategy.cpp:1103). `cells` receives one byte per block,
 * (strategy << 1) | anchor, the reference's AcStrategyGrid encoding
 * (src/core/ac_strategy.h:183-411). `costs` is the cost scratch above.
 */
GJXL_B200_API int gjxl_b200_ac_strategy_search(
    const float* opsin, size_t opsin_stride, size_t opsin_plane_pitch,
    size_t padded_width, size_t padded_height, const float* quant_field,
    const float* pixel_mask, size_t pixel_mask_stride, const int8_t* y_to_x,
    const int8_t* y_to_b, float butteraugli_target, int dense_dct32,
    int precision, float* costs, uint8_t* cells, uint32_t* device_error,
    void* stream);

/*
 * Butteraugli with a prepared reference image (rows a14, a15).
 * Replaces DeviceButteraugliOperation / PreparedDeviceButteraugli
 * (src/gpu/ops/butteraugli.h:53-150) as implemented by
 * LaunchCudaButteraugliPrepare / LaunchButteraugliCompareImpl
 * (src/gpu/cuda/cuda_butteraugli_kernels.cu:3927,3972), and the CPU
 * PreparedButteraugliReference::Prepare/Compare (src/codec/butteraugli.cpp:31,60).
 *
 * create() allocates all working planes for one extent (both scales);
 * prepare() transforms the reference once; compare() writes the distance map
 * (width x height, row stride map_stride) and, if `score` is non-null, the
 * maximum as a device double. Linear RGB inputs are 3 planes with the given
 * row stride and plane pitch. A handle serves one stream at a time.
 */
typedef struct gjxl_b200_butteraugli gjxl_b200_butteraugli;
GJXL_B200_API int gjxl_b200_butteraugli_create(size_t width, size_t height,
                                               float intensity_target,
                                               gjxl_b200_butteraugli** out);
GJXL_B200_API void gjxl_b200_butteraugli_destroy(gjxl_b200_butteraugli* b);
GJXL_B200_API int gjxl_b200_butteraugli_prepare(gjxl_b200_butteraugli* b,
                                                const float* reference,
                                                size_t stride,
                                                size_t plane_pitch,
                                                void* stream);
GJXL_B200_API int gjxl_b200_butteraugli_compare(
    gjxl_b200_butteraugli* b, const float* distorted, size_t stride,
    size_t plane_pitch, float* distance_map, size_t map_stride,
    double* score, uint32_t* device_error, void* stream);

/*
 * Global Butteraugli p-norm of a distance map (width x height floats, row
 * stride map_stride), accumulated in double precision: the mean of the p-,
 * 2p- and 4p-norms, ((S_p/n)^(1/p) + (S_2p/n)^(1/2p) + (S_4p/n)^(1/4p)) / 3
 * with S_q the sum of d^q over the n pixels (libjxl's published p-norm
 * summary; the reference summarises a map by its maximum only,
 * src/gpu/cuda/cuda_butteraugli_kernels.cu:4063-4065). Writes one device
 * double; fixed reduction order, so repeated calls agree to the bit.
 * `scratch`: device memory of gjxl_b200_butteraugli_pnorm_scratch_bytes().
 */
GJXL_B200_API size_t gjxl_b200_butteraugli_pnorm_scratch_bytes(void);
GJXL_B200_API int gjxl_b200_butteraugli_pnorm(const float* distance_map, size_t map_stride,
                                              size_t width, size_t height, double p,
                                              double* scratch, size_t scratch_bytes,
                                              double* pnorm, void* stream);

/* ------------------------------------------------------------------------
 * AC group packing, coefficient-order populations and AC tokenization
 * (rows a17, a18).
 *
 * Replaces the reference's AC-group packing and order-population kernels
 * (PackAcGroupsKernel cuda_ac_group_kernels.cu:13,
 * CoefficientOrderPopulationKernel cuda_coefficient_order_kernels.cu:29) and
 * the AcTokenizationProvider seam
 * (src/codestream/ac_tokenization_provider_internal.h:20-31) with the CPU
 * semantics of TokenizeSimpleAcGroupDirectValidated
 * (src/codestream/ac_group.cpp:740) and ComputeSimpleCoefficientOrdersForEncoder
 * (src/codestream/coefficient_order.cpp:568-830).
 *
 * Inputs: the strategy grid, the raw quant field (blocks) and quantized AC in
 * footprint layout (gjxl_b200_outputs). Tokens of every 256x256 group are
 * written back to back in row-major group order; group g's tokens are
 * token_values/contexts[group_offsets[g] .. group_offsets[g+1]). Within a
 * group: anchors in raster order, channels Y, X, B, each a nonzero-count token
 * followed by its coefficient tokens in scan order. order_mode: 0 natural
 * scans, 1 custom scans from full zero counts, 2 the effort-7 behaviour (DCT8
 * populations sampled when the frame holds DCT8 only).
 * ------------------------------------------------------------------------ */

typedef struct gjxl_b200_block_context_map {
  uint32_t threshold_count;          /* raw-quant thresholds, 0..15 */
  uint32_t qf_thresholds[15];
  uint32_t num_contexts;             /* 1..16 */
  /* [(channel_row * 13 + order_family) * (threshold_count + 1) + segment] */
  uint8_t context_map[3 * 13 * 16];
} gjxl_b200_block_context_map;

typedef struct gjxl_b200_ac_token_outputs {
  uint32_t* token_values;        /* required, token_capacity entries */
  uint16_t* token_contexts;      /* required, token_capacity entries */
  size_t token_capacity;         /* >= gjxl_b200_ac_token_capacity() */
  uint32_t* group_offsets;       /* required, groups + 1 */
  uint32_t* histogram;           /* optional: [num_contexts * 495][128] counts */
  int32_t* packed_ac;            /* optional: group order, 3 x 64 x blocks */
  uint32_t* group_coef_offsets;  /* optional: groups + 1 offsets into packed_ac */
  uint32_t* order_population;    /* optional: 6144 zero counts (3 x 1984 + 3 x 64) */
  uint32_t* present_mask;        /* optional device word: order families present */
  uint32_t* used_order_mask;     /* optional device word: families with custom scans */
  uint32_t* orders;              /* optional: [13][3][1024] scans in use */
  uint32_t* device_error;        /* optional */
} gjxl_b200_ac_token_outputs;

typedef struct gjxl_b200_ac_tokens gjxl_b200_ac_tokens;
GJXL_B200_API size_t gjxl_b200_ac_token_capacity(size_t blocks_x, size_t blocks_y);
GJXL_B200_API int gjxl_b200_ac_tokens_create(size_t blocks_x, size_t blocks_y,
                                             gjxl_b200_ac_tokens** out);
GJXL_B200_API void gjxl_b200_ac_tokens_destroy(gjxl_b200_ac_tokens* tokens);
GJXL_B200_API int gjxl_b200_ac_tokenize(
    gjxl_b200_ac_tokens* tokens, const uint8_t* strategy_cells,
    const int32_t* raw_quant_field, const int32_t* quantized_ac, size_t stride,
    size_t plane_pitch, const gjxl_b200_block_context_map* map, int order_mode,
    const gjxl_b200_ac_token_outputs* outputs, void* stream);

/* ------------------------------------------------------------------------
 * Analysis session: the whole analysis path for one image extent.
 *
 * Replaces the reference's prepared pipeline objects and their GPU providers:
 * PrepareResidentInput + PrepareResidentQuantizationPipeline +
 * RunPreparedGpuQuantizationPipelineForEncoding
 * (src/gpu/ops/resident_input.h:75-95,
 * src/codec/quantization_pipeline_internal.h:153-160,
 * src/gpu/ops/quantization_pipeline.cpp:970). A session owns all device
 * buffers for its extent (allocated once at creation) and enqueues every
 * stage on the caller's stream; independent sessions may run concurrently on
 * different streams, one session must not be used by two calls at once.
 * ------------------------------------------------------------------------ */

typedef struct gjxl_b200_options {
  size_t struct_size;       /* sizeof(gjxl_b200_options) */
  float butteraugli_target; /* distance; reference default 1.0 */
  int effort;               /* 5..10 (mixed-transform search); default 7 */
  float intensity_target;   /* XYB intensity target; the workflow uses 255 */
  int profile_stages;       /* nonzero: record CUDA events around each stage */
  int tokenize;             /* nonzero (default): AC tokens after the last evaluation */
  int order_mode;           /* -1 (default): by effort, as the reference resolves it
                               (effort 7: 2, else 1); or 0/1/2 as for
                               gjxl_b200_ac_tokenize */
  int precision;            /* GJXL_B200_PRECISION_EXACT (default) or _FAST:
                               candidate-cost precision of the strategy search */
  /* Learned mode (row N4; no reference counterpart). proposal_weights: device
   * pointer to gjxl_b200_cnn_param_count() FP32 parameters of the proposal
   * network, NULL (default) for the plain method. The network then proposes
   * three strategies per block: in a tile whose blocks all keep at least
   * proposal_confidence (default 0.6) of the probability mass on their
   * proposals, the greedy merge considers only the proposed families (and
   * DCT8); other tiles keep the full search. The refinement starts from the
   * adjusted field scaled by the predicted factor and runs
   * learned_iterations field updates (default 1; -1: the effort's) instead
   * of the effort's. */
  const float* proposal_weights;
  int learned_iterations;
  float proposal_confidence;
} gjxl_b200_options;

/* Session results. The adaptive-quantization fields mirror the reference's
 * CpuQuantizationPipelineOutput / VarDctEncoderFrame
 * (src/codec/quantization_pipeline.h, src/codec/vardct_frame.h) after the last
 * of the (iterations + 1) evaluations. Coefficient planes use "footprint
 * layout": the N coefficients of a transform anchored at block (bx, by) lie
 * in its own W x H pixel footprint, coefficient i at
 * (bx*8 + i % W, by*8 + i / W) of a padded plane; the reference's AC group
 * order is the anchors of each 256x256 group in raster order, each adding its
 * coefficients 0..N-1 per channel. */
typedef struct gjxl_b200_outputs {
  size_t padded_width, padded_height, blocks_x, blocks_y, tiles_x, tiles_y;
  size_t iterations;                /* evaluations - 1 */
  /* Device views (valid until the session is destroyed). */
  const float* linear;             /* 3 planes, unpadded */
  size_t linear_stride, linear_plane_pitch;
  const float* opsin;              /* padded XYB */
  const float* preprocessed_opsin; /* Gaborish-inverted XYB */
  size_t opsin_stride, opsin_plane_pitch;
  const float* initial_quant_field; /* blocks */
  const float* strategy_mask;       /* blocks */
  const float* pixel_mask;          /* padded pixels, stride opsin_stride */
  const int8_t* initial_y_to_x;     /* tiles, before the final CfL */
  const int8_t* initial_y_to_b;
  const uint8_t* strategy_cells;    /* blocks, (strategy << 1) | anchor */
  const float* matrix_scale_stats;  /* x_edge, b_edge, exposed_blue */
  const int* matrix_scales;         /* x_qm_scale, b_qm_scale */
  const float* quant_field;         /* blocks, final field */
  const float* adjusted_quant_field; /* blocks, the field the refinement starts from */
  /* Learned mode: per block the 3 proposed strategy codes, their softmax
   * mass and the predicted log field scale; per tile the searched families
   * (bit f: family f of DCT8, 16x8, 8x16, 16x16, 32x16, 16x32, 32x32). */
  const uint8_t* proposals;
  const float* proposal_mass;
  const float* proposal_log_scale;
  const uint8_t* tile_family_masks;
  const int32_t* raw_quant_field;   /* blocks */
  const int8_t* y_to_x;             /* tiles, final CfL map */
  const int8_t* y_to_b;
  const int32_t* quantized_ac;      /* 3 padded planes, footprint layout */
  const int32_t* quantized_dc;      /* 3 x blocks (X, Y, B) */
  const float* dc;                  /* 3 x blocks, dequantized DC */
  const float* block_distance;      /* blocks */
  const float* reconstructed_linear; /* 3 x width x height */
  const float* distance_map;        /* width x height */
  const double* score_history;      /* iterations + 1 maxima */
  const uint32_t* quantizer_params; /* global_scale, quant_dc, ... */
  const uint32_t* device_error;     /* [0] analysis, [1] Butteraugli, [2] tokens */
  /* Pinned host mirrors, filled by gjxl_b200_session_analyze_host once the
   * stream has completed. */
  const uint8_t* host_strategy_cells;
  const float* host_initial_quant_field;
  const int8_t* host_y_to_x;        /* final CfL map */
  const int8_t* host_y_to_b;
  const float* host_matrix_scale_stats;
  const uint32_t* host_device_error; /* 3 words */
  const float* host_quant_field;
  const int32_t* host_raw_quant_field;
  const int32_t* host_quantized_dc;
  const double* host_score_history;
  const uint32_t* host_quantizer_params;
  const int32_t* host_quantized_ac;
  /* AC tokens (tokenize != 0), with the reference's initial block-context
   * map (src/codestream/simple_ac_context.h:27-31): device views, then host
   * mirrors holding host_token_count tokens after
   * gjxl_b200_session_analyze_host. */
  size_t groups;
  const uint32_t* token_values;
  const uint16_t* token_contexts;
  const uint32_t* group_offsets;      /* groups + 1 */
  const uint32_t* token_histogram;    /* [4 * 495][128] */
  const uint32_t* scans;              /* [13][3][1024] coefficient scans in use */
  const uint32_t* order_masks;        /* present families, families with custom scans */
  const uint32_t* host_token_values;
  const uint16_t* host_token_contexts;
  const uint32_t* host_group_offsets;
  size_t host_token_count;
  size_t device_bytes;
  /* The session's own input buffer (packed rows of width * channels bytes,
   * input_capacity bytes): a device-resident caller that writes its image
   * here and passes this pointer to gjxl_b200_session_analyze saves the
   * input copy. */
  uint8_t* input_pixels;
  size_t input_capacity;
  int graph_replay;                 /* 1 once analyses replay a captured graph */
  /* FP64 global Butteraugli p-norm (p = 3, gjxl_b200_butteraugli_pnorm) of
   * each evaluation's distance map, iterations + 1 values: device, then the
   * host mirror filled by gjxl_b200_session_analyze_host. */
  const double* pnorm_history;
  const double* host_pnorm_history;
  /* DC-group token streams (tokenize != 0), gjxl_b200_dc_tokenize's layout
   * with the weighted DC predictor and default EPF sharpness: DC residual
   * tokens (3 * blocks pairs, written by the last DC quantization),
   * AC-metadata tokens, the per-group table (5 words per group) and the
   * [45][128] histogram. Device views, then host mirrors filled by
   * gjxl_b200_session_analyze_host (host_meta_token_count pairs). */
  size_t dc_groups;
  const uint32_t* dc_tokens;
  const uint32_t* meta_tokens;
  const uint32_t* dc_group_info;
  const uint32_t* dc_histogram;
  const uint32_t* host_dc_tokens;
  const uint32_t* host_meta_tokens;
  const uint32_t* host_dc_group_info;
  const uint32_t* host_dc_histogram;
  size_t host_meta_token_count;
} gjxl_b200_outputs;

typedef struct gjxl_b200_session gjxl_b200_session;

GJXL_B200_API void gjxl_b200_default_options(gjxl_b200_options* options);
GJXL_B200_API int gjxl_b200_session_create(size_t width, size_t height,
                                           const gjxl_b200_options* options,
                                           gjxl_b200_session** session);
GJXL_B200_API void gjxl_b200_session_destroy(gjxl_b200_session* session);
/* Device bytes a session of this extent and options needs for its working
 * buffers (all but a small per-session table of the AC tokenizer), and a
 * session whose working buffers are carved from caller memory (256-byte
 * aligned, at least that many bytes; not freed by the session). Sessions
 * that never run at the same time, such as those of one batch lane, may
 * share one region: nothing in it outlives an analysis. Pinned host mirrors
 * are allocated by a session's first gjxl_b200_session_analyze_host. */
GJXL_B200_API int gjxl_b200_session_device_bytes(size_t width, size_t height,
                                                 const gjxl_b200_options* options,
                                                 size_t* bytes);
GJXL_B200_API int gjxl_b200_session_create_in(size_t width, size_t height,
                                              const gjxl_b200_options* options,
                                              void* device_memory, size_t device_bytes,
                                              gjxl_b200_session** session);
/* Changes the Butteraugli target of later analyses, keeping every buffer of
 * the session (the prepared state a target-size search reuses across its
 * attempts: src/codestream/workflow.cpp:1686-1740, rate_control.cpp:246).
 * The next analysis captures its graph again. */
GJXL_B200_API int gjxl_b200_session_set_butteraugli_target(gjxl_b200_session* session,
                                                           float butteraugli_target);
/* Device-resident input: packed 8-bit sRGB already in device memory. The
 * first call for a channel count captures the analysis into a CUDA graph
 * over the session's input buffer; later calls replay it. Input anywhere
 * else is first copied into that buffer on `stream` (no recapture when the
 * pointer changes). Asynchronous: read outputs.device_error (or call
 * gjxl_b200_check_device_error) once the stream has completed. */
GJXL_B200_API int gjxl_b200_session_analyze(gjxl_b200_session* session,
                                            const uint8_t* pixels,
                                            size_t row_stride_bytes,
                                            int channels, void* stream);
/* Host input: one host-to-device copy of the packed pixels, the analysis,
 * and device-to-host copies of the results into the host mirrors. Returns
 * once the stream has completed and the mirrors are filled (the token count
 * is known only then); returns GJXL_B200_DEVICE_ERROR when a device error
 * word is set. */
GJXL_B200_API int gjxl_b200_session_analyze_host(gjxl_b200_session* session,
                                                 const uint8_t* host_pixels,
                                                 size_t row_stride_bytes,
                                                 int channels, void* stream);
GJXL_B200_API int gjxl_b200_session_outputs(const gjxl_b200_session* session,
                                            gjxl_b200_outputs* outputs);
/* Per-stage milliseconds of the last analysis (profile_stages only; call
 * after the stream completed). Returns the number of stages written. */
GJXL_B200_API int gjxl_b200_session_stage_times(gjxl_b200_session* session,
                                                float* milliseconds,
                                                int capacity);
GJXL_B200_API const char* gjxl_b200_stage_name(int stage);
/* Number of kernels one gjxl_b200_session_analyze call on these arguments
 * launches: the analysis is captured into a CUDA graph on a private stream
 * (nothing executes) and its kernel nodes are counted. Needs a session
 * created with profile_stages off. No counterpart in the reference. */
GJXL_B200_API int gjxl_b200_session_kernel_count(gjxl_b200_session* session,
                                                 const uint8_t* pixels,
                                                 size_t row_stride_bytes, int channels,
                                                 size_t* kernels);

/*
 * Batched analysis (row N3). Replaces the reference's VarDctBatchEncoder
 * (src/codestream/batch_workflow.h:74-118) for the analysis half: one call
 * runs every request, keeps request order in the results, reports a status
 * per image and times each image as queue / service / ready (milliseconds
 * from the batch's arrival, device clock). Each image runs its own session
 * (pooled per extent and reused by later calls, so a repeated batch replays
 * captured graphs) on one of `lanes` CUDA streams; the lanes' analyses run
 * concurrently. max_in_flight: lanes, 1..16 (0: 2 until autotuned).
 */
typedef struct gjxl_b200_batch gjxl_b200_batch;
typedef struct gjxl_b200_batch_request {
  const uint8_t* pixels;   /* packed 8-bit sRGB rows: device memory, or host
                              memory when host_input is set */
  size_t width, height, row_stride;
  int channels;            /* 3 or 4 */
  float butteraugli_target;
} gjxl_b200_batch_request;
typedef struct gjxl_b200_batch_result {
  int status;                   /* StatusCode of this image */
  gjxl_b200_session* session;   /* its results: gjxl_b200_session_outputs */
  int lane;
  double queue_ms, service_ms, ready_ms;
} gjxl_b200_batch_result;

GJXL_B200_API int gjxl_b200_batch_create(int max_in_flight, const gjxl_b200_options* options,
                                         gjxl_b200_batch** batch);
GJXL_B200_API void gjxl_b200_batch_destroy(gjxl_b200_batch* batch);
/* Lanes and order (0: as given, 1: largest first) of later calls. */
GJXL_B200_API int gjxl_b200_batch_set_schedule(gjxl_b200_batch* batch, int lanes,
                                               int largest_first);
/* Runs the batch and waits for it. host_input: pixels are host memory and
 * each image goes through gjxl_b200_session_analyze_host (host mirrors
 * filled), one host thread per lane; else device memory and
 * gjxl_b200_session_analyze. batch_ms: arrival to the last image's end. */
GJXL_B200_API int gjxl_b200_batch_analyze(gjxl_b200_batch* batch,
                                          const gjxl_b200_batch_request* requests,
                                          size_t count, int host_input,
                                          gjxl_b200_batch_result* results, double* batch_ms);
/* Autotuner: runs the (device-input) batch with each lane count of
 * lane_counts and both orders, keeps the fastest and returns it. */
GJXL_B200_API int gjxl_b200_batch_autotune(gjxl_b200_batch* batch,
                                           const gjxl_b200_batch_request* requests,
                                           size_t count, const int* lane_counts,
                                           size_t lane_count_count, int* lanes,
                                           int* largest_first);
/* The placement rule (host only): order[k] = k-th request to place (as
 * given, or by decreasing pixels, ties in request order); each goes to the
 * lane with the fewest pixels so far (lowest index on ties). */
GJXL_B200_API int gjxl_b200_batch_schedule(size_t count, const size_t* pixels, int lanes,
                                           int largest_first, int* lane_of, size_t* order);
GJXL_B200_API size_t gjxl_b200_batch_device_bytes(const gjxl_b200_batch* batch);

/*
 * Measurement (no counterpart in the reference).
 * FP64 multiply/add throughput of the current device in operations per
 * second (one DMUL or DADD = one operation), measured with independent
 * separately rounded multiply-add chains: the ceiling of the bit-exact
 * double-precision transform kernels. `device_sink` is 8 bytes of device
 * memory (never written in practice). Synchronizes `stream`.
 */
GJXL_B200_API int gjxl_b200_fp64_throughput(double* device_sink, double* ops_per_second,
                                            void* stream);

/*
 * Reads `words` device error words (1..64) once `stream` has completed and
 * returns GJXL_B200_DEVICE_ERROR if any is nonzero. Replaces the reference's
 * ReadAndCheckDeviceError (src/gpu/cuda/cuda_aq_resident.cpp:3451).
 */
GJXL_B200_API int gjxl_b200_check_device_error(const uint32_t* device_error, size_t words,
                                               void* stream);

/*
 * Deterministic failure injection for tests, per calling thread. Replaces
 * the reference's CudaBackendOptions::test_fail_submission and
 * ArmNextCudaSubmissionFailureForTest (src/gpu/cuda/cuda_backend.h:19-21,60).
 * Arms the `check_point`-th (1-based) next check point of `kind` to fail
 * (0 disarms):
 *   1 allocation: a device or pinned host allocation in session, Butteraugli
 *     or token-handle creation fails with GJXL_B200_OUT_OF_MEMORY, and the
 *     handle releases what it had allocated;
 *   2 graph: the next graph instantiation fails; the session falls back to
 *     launching its stages directly;
 *   3 submission: the next session analysis fails with
 *     GJXL_B200_SUBMISSION_FAILED before anything is enqueued, leaving
 *     every output unchanged.
 * Failures are made on the host; nothing faults on the device.
 */
GJXL_B200_API int gjxl_b200_test_arm_failure(int kind, int check_point);

/*
 * Entropy-coded sections on the device: the token streams of many sections
 * (AC groups, DC groups, ...) written with an already built entropy code,
 * ANS or prefix, bit for bit as the reference's CPU writers write them.
 * Replaces WriteValidatedTokenStream (src/codestream/entropy.cpp:29), which
 * dispatches to WriteAnsTokenStream (src/codestream/ans.cpp:2305: the
 * reverse rANS recurrence of ans.cpp:1700-1770 and the reverse-bit append of
 * src/codestream/ans_reverse_bits_internal.h) or to the prefix
 * WriteTokenStream (src/codestream/entropy.cpp:2294, WriteValue :1173), as
 * WriteAcSections calls it once per AC group on its worker threads
 * (src/codestream/vardct/encoder.cpp:721-790); and the exact token-bit
 * counters CountAnsTokenStreamBits / MeasureAnsCodes (ans.cpp:1774,1875).
 * Model construction (clustering, normalisation, serialisation of the
 * histograms) stays with the caller, as in the reference.
 *
 * An EntropyCode (src/codestream/entropy.h:153) flattened into device tables:
 */
#define GJXL_B200_ENTROPY_PREFIX 0
#define GJXL_B200_ENTROPY_ANS 1
typedef struct gjxl_b200_entropy_code {
  int mode;                       /* GJXL_B200_ENTROPY_PREFIX or _ANS */
  uint32_t context_count;         /* 1..65536 */
  uint32_t cluster_count;         /* 1..256 */
  const uint8_t* context_map;     /* [context_count]: cluster of each context */
  const uint8_t* uint_configs;    /* [cluster_count][3]: HybridUintConfig
                                     {split_exponent, msb_in_token, lsb_in_token} */
  /* Prefix codes (mode 0), PrefixCode per cluster over 128 symbols. */
  const uint8_t* prefix_depths;   /* [cluster][128]: code length, 0 = absent */
  const uint16_t* prefix_bits;    /* [cluster][128]: code bits, first bit in bit 0 */
  const uint16_t* prefix_degenerate; /* [cluster]: the symbol written with no
                                        bits (degenerate_symbol), 128 = none */
  /* ANS (mode 1), AnsHistogram per cluster over 256 symbols of a 4096 table. */
  const uint16_t* ans_frequencies;      /* [cluster][256]: 0 = absent */
  const uint16_t* ans_reverse_offsets;  /* [cluster][256]: prefix sums of the frequencies */
  const uint16_t* ans_reverse_map;      /* [cluster][4096] */
} gjxl_b200_entropy_code;

/*
 * Token streams of `count` sections. Tokens are EntropyToken {context, value}
 * either interleaved (`pairs`: context, value uint32 pairs, the DC-group and
 * metadata token layout) or split (`values` uint32 + `contexts` uint16, the
 * AC token layout of gjxl_b200_ac_tokenize), all device memory. Section s
 * holds tokens offsets[s] .. offsets[s + 1] - 1 (device uint32[count + 1]).
 */
typedef struct gjxl_b200_token_sections {
  const uint32_t* pairs;
  const uint32_t* values;
  const uint16_t* contexts;
  const uint32_t* offsets;
  uint32_t count;
  uint32_t capacity;  /* tokens the arrays hold: a section reaching past it
                         sets device_error bit 2 and is not read */
} gjxl_b200_token_sections;

/*
 * Words of the slot buffer gjxl_b200_entropy_write_sections needs for
 * `sections` sections of `tokens` tokens in all (47 bits per ANS token plus
 * its 32-bit final state, 46 per prefix token, two words per section).
 * Section s's slot starts at word ceil(B * offsets[s] / 64) + 2 s
 * (B = 47 for ANS, 46 for prefix).
 */
GJXL_B200_API size_t gjxl_b200_entropy_slot_words(int mode, size_t tokens, size_t sections);

/*
 * Writes every section's token stream with `code` (host struct of device
 * tables), ANS or prefix. Each section is written from bit 0 of its slot in
 * `slot_words` (little-endian 64-bit words, first bit in bit 0, the
 * reference BitWriter's byte order) and its length goes to bit_counts[s]
 * (device uint64[count]) — BitWriter::bits_written() of the reference's
 * section. With `packed` non-NULL the sections are also concatenated, each
 * zero-padded to a byte boundary (BitWriter::padded_bytes()), in section
 * order, and byte_offsets (device uint64[count + 1]) receives each section's
 * first byte and the total: the codestream's section bytes in TOC order.
 * packed_capacity >= 8 * slot_word_capacity always suffices. A token whose
 * context is out of range or whose symbol the code lacks sets device_error
 * bit 2 (the reference's InvalidArgument); that section's output is then
 * undefined.
 */
GJXL_B200_API int gjxl_b200_entropy_write_sections(
  const gjxl_b200_entropy_code* code, const gjxl_b200_token_sections* sections,
  uint64_t* slot_words, size_t slot_word_capacity, uint64_t* bit_counts, uint8_t* packed,
  size_t packed_capacity, uint64_t* byte_offsets, uint32_t* device_error, void* stream);

/*
 * Exact token-stream bits of every section under each of `code_count`
 * (1..8) codes (host array of structs of device tables): bit_counts[s *
 * code_count + c] (device uint64) equals CountAnsTokenStreamBits (ANS: 32 +
 * extra bits + 16 per renormalisation) or the prefix stream's length, the
 * figures MeasureAnsCodes and the rate search compare (ans.cpp:1875). Errors
 * as gjxl_b200_entropy_write_sections.
 */
GJXL_B200_API int gjxl_b200_entropy_count_sections(
  const gjxl_b200_entropy_code* codes, uint32_t code_count,
  const gjxl_b200_token_sections* sections, uint64_t* bit_counts, uint32_t* device_error,
  void* stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* GJXL_B200_H_ */
