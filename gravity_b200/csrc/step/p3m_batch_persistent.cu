// p3m_batch_persistent.cu — the batched form's step as ONE persistent launch.
//
// The fused batch (p3m_api.cu, build_fused) describes a batch step as a list
// of stages; each stage is one of the batched bodies below over all the
// simulations it concerns (virtual block b of a stage is local block
// b - first[s] of simulation s). Here those stages run inside one
// cooperative kernel with every CTA resident: the stages are grouped into
// phases (stages of a phase are independent, e.g. the short range beside the
// FFT rows), the CTAs stride over a phase's virtual blocks, and a grid
// barrier separates the phases.
//
// The barrier is bounded: a CTA polls the arrival counter at most
// `poll_limit` times (with a short sleep), then counts the wait as given up
// in sync[1] and ends; a CTA that did not get past a barrier never runs the
// stages behind it, so no stage ever reads the output of an unfinished one.
// The host reports the count as P3M_ERR_TIMEOUT. A test hook makes one CTA
// skip its arrival at one phase (as a CTA that never arrives would).
//
// Stage outputs are read by other SMs within the same launch, so the bodies
// used here are the coherent copy of the stage sources (namespace
// p3m::coherent, compiled without the read-only non-coherent load path),
// which p3m_step.cu includes before this file.

namespace p3m {
namespace {

__device__ __forceinline__ unsigned int load_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Exclusive prefix sum of one radix histogram of at most kPersistentScanMax
// words by a 256-thread CTA (the persistent kernel's form of the scan that
// the multi-launch batch runs with 1024 threads).
constexpr int kPersistentScanItems = 32;
constexpr int kPersistentScanMax = 256 * kPersistentScanItems;

__device__ __forceinline__ void scan256_body(uint32_t* data, int n, uint32_t* warp_tot) {
    const int base = threadIdx.x * kPersistentScanItems;
    uint32_t v[kPersistentScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kPersistentScanItems; ++i) {
        v[i] = base + i < n ? data[base + i] : 0u;
        s += v[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t pre = inc - s;
    for (int w = 0; w < warp; ++w) pre += warp_tot[w];
#pragma unroll
    for (int i = 0; i < kPersistentScanItems; ++i) {
        if (base + i < n) data[base + i] = pre;
        pre += v[i];
    }
}

// Every stage kind's virtual block, each out of line (one function per
// kind, no branch on the kind inside): registers are then allocated for each
// body on its own, under the kernel's budget, instead of for all at once.
namespace C = coherent::p3m;
#define P3M_STAGE(name) \
    __device__ __noinline__ void name(int2 sb, const unsigned char* args, const float2* tw, unsigned char* pool)

P3M_STAGE(stage_morton) {
    const MortonArgs a = reinterpret_cast<const MortonArgs*>(args)[sb.x];
    C::morton_keys_body(sb.y, a.bodies, a.n, a.wbits, a.hbits, a.keys, a.vals);
}
P3M_STAGE(stage_radix_hist) {
    const RadixArgs a = reinterpret_cast<const RadixArgs*>(args)[sb.x];
    C::radix_hist_body(sb.y, a.keys_in, a.n, a.shift, a.bits, a.tiles, a.hist);
}
P3M_STAGE(stage_scan) {
    const ScanArgs a = reinterpret_cast<const ScanArgs*>(args)[sb.x];
    scan256_body(a.data, a.n, reinterpret_cast<uint32_t*>(pool));
}
P3M_STAGE(stage_radix_scatter) {
    const RadixArgs a = reinterpret_cast<const RadixArgs*>(args)[sb.x];
    C::radix_scatter_body<false, kSortMaxRadix>(
        *reinterpret_cast<C::ScatterShared<kSortMaxRadix>*>(pool), sb.y, a.keys_in, a.vals_in,
        a.keys_out, a.vals_out, a.n, a.shift, a.bits, a.tiles, a.hist);
}
P3M_STAGE(stage_permute) {
    const PermuteArgs a = reinterpret_cast<const PermuteArgs*>(args)[sb.x];
    C::permute_body(sb.y, a.order, a.n, a.bodies, a.accel, a.materials, a.bodies_out, a.accel_out,
                    a.materials_out, a.destinations);
}
P3M_STAGE(stage_copy) {
    const CopyArgs a = reinterpret_cast<const CopyArgs*>(args)[sb.x];
    const long long i = (long long)sb.y * blockDim.x + threadIdx.x;
    if (i < a.words) a.dst[i] = a.src[i];
}
P3M_STAGE(stage_drift) {
    const DriftArgs a = reinterpret_cast<const DriftArgs*>(args)[sb.x];
    C::drift_body(sb.y, a.bodies, a.accel, a.n, a.half_kick, a.drift_dt, a.substeps, a.bounded,
                  a.W, a.H, a.keys, a.vals, a.nonfinite);
}
P3M_STAGE(stage_zero) {
    const ZeroArgs a = reinterpret_cast<const ZeroArgs*>(args)[sb.x];
    const long long base = (long long)sb.y * (kBatchThreads * 16);
    for (int i = threadIdx.x; i < kBatchThreads * 16; i += blockDim.x) {
        const long long w = base + i;
        if (w < a.words) a.data[w] = 0u;
    }
}
P3M_STAGE(stage_cell_build) {
    const CellBuildArgs a = reinterpret_cast<const CellBuildArgs*>(args)[sb.x];
    C::cell_build_body(sb.y, a.keys, a.ids, a.n, a.bodies, a.materials, a.cell_start,
                       a.cell_count, a.cell_mass, a.entries, 0);
}
P3M_STAGE(stage_slots) {
    const SlotsArgs a = reinterpret_cast<const SlotsArgs*>(args)[sb.x];
    C::cell_slots_body(sb.y, a.cell_start, a.cell_count, a.cell_mass, a.entries, a.W, a.H,
                       a.gravity, a.total_mass, a.slots);
}
P3M_STAGE(stage_short_range_slots) {
    const ShortRangeArgs a = reinterpret_cast<const ShortRangeArgs*>(args)[sb.x];
    C::sr::short_range_body<kPersistentRx, kPersistentRy, 2>(
        reinterpret_cast<C::sr::SlotStage*>(pool), sb.y, a.bodies, a.entries, a.cell_start,
        a.cell_count, a.cell_mass, a.slots, a.a_short, a.p);
}
P3M_STAGE(stage_short_range_lists) {
    const ShortRangeArgs a = reinterpret_cast<const ShortRangeArgs*>(args)[sb.x];
    C::sr::short_range_body<kPersistentRx, kPersistentRy, 0>(
        nullptr, sb.y, a.bodies, a.entries, a.cell_start, a.cell_count, a.cell_mass, a.slots,
        a.a_short, a.p);
}
P3M_STAGE(stage_deposit_i64) {
    const DepositArgs a = reinterpret_cast<const DepositArgs*>(args)[sb.x];
    C::deposit_chunks_body<unsigned long long>(sb.y, a.entries, a.keys, a.n, a.W, a.H, a.MW, a.MH,
                                               a.scale, static_cast<unsigned long long*>(a.density),
                                               C::kWindowBytes / 8);
}
P3M_STAGE(stage_deposit_u32) {
    const DepositArgs a = reinterpret_cast<const DepositArgs*>(args)[sb.x];
    C::deposit_chunks_body<uint32_t>(sb.y, a.entries, a.keys, a.n, a.W, a.H, a.MW, a.MH, a.scale,
                                     static_cast<uint32_t*>(a.density), C::kWindowBytes / 4);
}
P3M_STAGE(stage_fft_rows_i64) {
    const FftRowsArgs a = reinterpret_cast<const FftRowsArgs*>(args)[sb.x];
    C::fft_rows_forward_body<long long>(sb.y, static_cast<const long long*>(a.density), a.inv_scale,
                                        a.MW, a.MH, a.per_cta, tw, a.half);
}
P3M_STAGE(stage_fft_rows_u32) {
    const FftRowsArgs a = reinterpret_cast<const FftRowsArgs*>(args)[sb.x];
    C::fft_rows_forward_body<uint32_t>(sb.y, static_cast<const uint32_t*>(a.density), a.inv_scale,
                                       a.MW, a.MH, a.per_cta, tw, a.half);
}
P3M_STAGE(stage_fft_columns) {
    const FftColumnsArgs a = reinterpret_cast<const FftColumnsArgs*>(args)[sb.x];
    C::fft_columns_body(sb.y, a.half, a.green, a.inv_total, a.MW, a.MH, a.per_cta, tw, a.cols);
}
P3M_STAGE(stage_fft_inverse) {
    const FftInverseArgs a = reinterpret_cast<const FftInverseArgs*>(args)[sb.x];
    C::fft_rows_inverse_body(sb.y, a.cols, a.MW, a.MH, a.per_cta, tw, a.force);
}
P3M_STAGE(stage_kick) {
    const KickArgs a = reinterpret_cast<const KickArgs*>(args)[sb.x];
    C::interp_kick_body(sb.y, a.bodies, a.accel, a.force, a.a_short, a.p);
}
#undef P3M_STAGE

// Whether a stage kind uses the CTA's shared memory (then the CTA's next
// virtual block may only start after a barrier).
__device__ __forceinline__ bool stage_uses_shared(int kind) {
    switch (kind) {
        case kPStageRadixHist: case kPStageScan: case kPStageRadixScatter:
        case kPStageShortRangeSlots: case kPStageDepositU32: case kPStageDepositI64:
        case kPStageFftRowsU32: case kPStageFftRowsI64: case kPStageFftColumns:
        case kPStageFftInverse:
            return true;
        default:
            return false;
    }
}

// One virtual block of one stage: local block sb.y of simulation sb.x.
__device__ __forceinline__ void run_stage(int kind, int2 sb, const unsigned char* args,
                                          const float2* tw, unsigned char* pool) {
    switch (kind) {
        case kPStageMorton: stage_morton(sb, args, tw, pool); break;
        case kPStageRadixHist: stage_radix_hist(sb, args, tw, pool); break;
        case kPStageScan: stage_scan(sb, args, tw, pool); break;
        case kPStageRadixScatter: stage_radix_scatter(sb, args, tw, pool); break;
        case kPStagePermute: stage_permute(sb, args, tw, pool); break;
        case kPStageCopy: stage_copy(sb, args, tw, pool); break;
        case kPStageDrift: stage_drift(sb, args, tw, pool); break;
        case kPStageZero: stage_zero(sb, args, tw, pool); break;
        case kPStageCellBuild: stage_cell_build(sb, args, tw, pool); break;
        case kPStageSlots: stage_slots(sb, args, tw, pool); break;
        case kPStageShortRangeSlots: stage_short_range_slots(sb, args, tw, pool); break;
        case kPStageShortRangeLists: stage_short_range_lists(sb, args, tw, pool); break;
        case kPStageDepositU32: stage_deposit_u32(sb, args, tw, pool); break;
        case kPStageDepositI64: stage_deposit_i64(sb, args, tw, pool); break;
        case kPStageFftRowsU32: stage_fft_rows_u32(sb, args, tw, pool); break;
        case kPStageFftRowsI64: stage_fft_rows_i64(sb, args, tw, pool); break;
        case kPStageFftColumns: stage_fft_columns(sb, args, tw, pool); break;
        case kPStageFftInverse: stage_fft_inverse(sb, args, tw, pool); break;
        case kPStageKick: stage_kick(sb, args, tw, pool); break;
        default: break;
    }
}

// Bounded grid barrier after `phase`: sync[0] counts arrivals over the whole
// launch (cleared before it), sync[1] the waits that gave up. Returns false
// (in every thread of the CTA) when this CTA must end.
__device__ __forceinline__ bool grid_barrier(unsigned int* sync, int phase, int poll_limit,
                                             bool withhold, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 0;
        if (!withhold) {
            __threadfence();
            atomicAdd(&sync[0], 1u);
            const unsigned int target = (unsigned int)(phase + 1) * gridDim.x;
            ok = 1;
            int polls = 0;
            while (load_acquire(&sync[0]) < target) {
                if (++polls > poll_limit) {
                    atomicAdd(&sync[1], 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// phase_ns (when not null): CTA 0 records the global timer at the start and
// as it leaves each phase's barrier (n_phases + 1 stamps, at most
// kPersistentMaxStamps), the per-phase profile of the last launch.
__global__ void __launch_bounds__(kBatchThreads, 2) batch_persistent_kernel(
    const unsigned char* __restrict__ blob, const PStage* __restrict__ stages,
    const PPhase* __restrict__ phases, int n_phases, const float2* tw, unsigned int* sync,
    int poll_limit, int withhold_cta, int withhold_phase, unsigned long long* phase_ns) {
    extern __shared__ __align__(16) unsigned char p3m_pool[];
    __shared__ int s_ok;
    const bool stamp = phase_ns != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
    if (stamp) phase_ns[0] = global_ns();
    for (int ph = 0; ph < n_phases; ++ph) {
        const PPhase P = phases[ph];
        int total = 0;
        for (int k = 0; k < P.stages; ++k) total += stages[P.first_stage + k].blocks;
        // The CTA's virtual blocks increase, so its stage and simulation are
        // found by moving two cursors forward (no search per block).
        int k = P.first_stage, base = 0, sim = 0;
        for (int v = blockIdx.x; v < total; v += gridDim.x) {
            while (v >= base + stages[k].blocks) {
                base += stages[k].blocks;
                ++k;
                sim = 0;
            }
            const PStage st = stages[k];
            const int local = v - base;
            const int* first = reinterpret_cast<const int*>(blob + st.first);
            while (sim + 1 < st.sims && first[sim + 1] <= local) ++sim;
            run_stage(st.kind, make_int2(sim, local - first[sim]), blob + st.args, tw, p3m_pool);
            if (stage_uses_shared(st.kind)) __syncthreads();  // the pool is reused next
        }
        if (ph + 1 == n_phases) {  // the stream orders the next launch
            if (stamp && ph + 1 < kPersistentMaxStamps) {
                __syncthreads();
                phase_ns[ph + 1] = global_ns();
            }
            break;
        }
        const bool withhold = (int)blockIdx.x == withhold_cta && ph == withhold_phase;
        if (!grid_barrier(sync, ph, poll_limit, withhold, &s_ok)) return;
        if (stamp && ph + 1 < kPersistentMaxStamps) phase_ns[ph + 1] = global_ns();
    }
}

}  // namespace

// Dynamic shared memory every persistent step needs besides its FFT stages':
// the scatter tile, the slot stage and the deposit window.
size_t persistent_base_smem() {
    size_t s = sizeof(coherent::p3m::ScatterShared<kSortMaxRadix>);
    if (sizeof(coherent::p3m::sr::SlotStage) > s) s = sizeof(coherent::p3m::sr::SlotStage);
    if ((size_t)coherent::p3m::kWindowBytes > s) s = (size_t)coherent::p3m::kWindowBytes;
    return s;
}

int persistent_scan_limit() { return kPersistentScanMax; }

// CTAs per SM the persistent kernel can keep resident with `smem` dynamic
// shared memory (0: it cannot run); sets the kernel's shared memory limit.
int persistent_ctas_per_sm(size_t smem) {
    if (cudaFuncSetAttribute(batch_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent_kernel,
                                                      kBatchThreads, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

cudaError_t launch_batch_persistent(const unsigned char* blob, const PStage* stages,
                                    const PPhase* phases, int n_phases, const float2* tw,
                                    unsigned int* sync, int poll_limit, int withhold_cta,
                                    int withhold_phase, int ctas, size_t smem,
                                    unsigned long long* phase_ns, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(sync, 0, sizeof(unsigned int), stream);  // arrivals
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, batch_persistent_kernel, blob, stages, phases, n_phases, tw, sync,
                           poll_limit, withhold_cta, withhold_phase, phase_ns);
    count_launches(1);
    return e;
}

}  // namespace p3m
