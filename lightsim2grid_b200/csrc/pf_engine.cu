// Batched AC Newton-Raphson on the GPU: one persistent kernel, one CTA per instance.
//
// Each CTA takes jobs (an instance, or a chain of time-series steps) from a global
// counter and runs the whole Newton loop of the reference's compute_pf for them:
//   mismatch   F = V .* conj(Ybus V) - Sbus (+ slack term)     BaseAlgo.cpp:30-118
//   J fill     dS/dVm, dS/dVa scattered into the LU array      BaseNRAlgo.tpp:202-260,
//                                                              BaseNRSingleSlackAlgo.tpp:449-490
//   refactor   LU with the plan's fixed pivots                 (KLUSolver.cpp:47-59 contract)
//   solve      forward / backward substitution                 (KLUSolver.cpp:61-69 contract)
//   update     Va, Vm, V and the convergence test              BaseNRSingleSlackAlgo.tpp:129-162,
//                                                              BaseNRAlgo.tpp:136-167
// Refactorisation: right-looking by elimination level; the update groups (pivot c, column j)
// of a level are spread over the CTA's threads in conflict-free phases, one barrier per
// phase, no atomics, so the result is deterministic.  Solves: row oriented and level
// scheduled with 1..32 lanes per row; levels with one or two rows run as a chain on warp 0
// with the next row's indices prefetched.  LU values live in shared memory when they fit,
// else in the CTA's global slab (L2 resident).  The mixed form (FP32 LU) refines every
// Newton step once against the FP64 Jacobian, computed on the fly from dS/dV.
#include "pf_engine.cuh"

namespace l2g {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cabs2(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v, int width) {
    for (int o = width >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, width);
    return v;
}

struct Shared {
    double red[32];
    int ired[32];
    int opos[kMaxOverrides];
    double2 oval[kMaxOverrides];
    int novr;
    int job;
    int piv_err;
    double slack_absorbed;
};

// block-wide max of |F| and "any non-finite" flag; every thread receives the result
__device__ __forceinline__ void block_norm(Shared &S, double lmax, int lbad, double &norm, int &bad) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        lbad |= __shfl_xor_sync(0xffffffffu, lbad, o);
    }
    __syncthreads();
    if (lane == 0) {
        S.red[warp] = lmax;
        S.ired[warp] = lbad;
    }
    __syncthreads();
    double r = 0.0;
    int b = 0;
    for (int w = 0; w < nw; ++w) {
        r = fmax(r, S.red[w]);
        b |= S.ired[w];
    }
    norm = r;
    bad = b;
}

__device__ __forceinline__ double block_min(Shared &S, double v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) S.red[warp] = v;
    __syncthreads();
    double r = S.red[0];
    for (int w = 1; w < nw; ++w) r = fmin(r, S.red[w]);
    return r;
}

__device__ __forceinline__ double block_sum(Shared &S, double v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) S.red[warp] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < nw; ++w) r += S.red[w];
    return r;
}

__device__ __forceinline__ double2 ybus_value(const DevPlan &P, const Shared &S, int p) {
    double2 y = P.Rx[p];
    for (int i = 0; i < S.novr; ++i)
        if (S.opos[i] == p) y = S.oval[i];
    return y;
}

// dS/dVa and dS/dVm of Ybus entry (r, c), as BaseNRAlgo::_dSbus_dV (BaseNRAlgo.tpp:228-257)
__device__ __forceinline__ void dsbus(double2 y, double2 vr, double2 vc, bool diag, double2 ib, double &dvar,
                                      double &dvai, double2 &dvm) {
    const double ic = 1.0 / cabs2(vc);
    const double2 vnc = make_double2(vc.x * ic, vc.y * ic);
    double2 a = cmul(cconj(cmul(y, vnc)), vr);  // conj(Y * Vnorm_c) * V_r
    double2 b = cmul(y, vc);                    // Y * V_c
    if (diag) {
        const double ir = 1.0 / cabs2(vr);
        const double2 vnr = make_double2(vr.x * ir, vr.y * ir);
        const double2 t = cmul(cconj(ib), vnr);
        a.x += t.x;
        a.y += t.y;
        b.x -= ib.x;
        b.y -= ib.y;
    }
    dvar = b.x * vr.y - b.y * vr.x;  // conj(-b) * (j V_r)
    dvai = -(b.x * vr.x + b.y * vr.y);
    dvm = a;
}

// F at V: writes Ibus, the FP64 mismatch per bus and the permuted right-hand side x;
// returns ||F||_inf and a non-finite flag to every thread.
template <typename XT>
__device__ void mismatch(const DevPlan &P, Shared &S, const double2 *__restrict__ V, double2 *__restrict__ Ibus,
                         double2 *__restrict__ Fbus, const double2 *__restrict__ Sbus, XT *x, double &norm,
                         int &bad) {
    double lmax = 0.0;
    int lbad = 0;
    const double sa = S.slack_absorbed;
    for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        const int p1 = P.Rp[r + 1];
        for (int p = P.Rp[r]; p < p1; ++p) {
            const double2 y = ybus_value(P, S, p);
            const double2 v = V[P.Rj[p]];
            s.x += y.x * v.x - y.y * v.y;
            s.y += y.x * v.y + y.y * v.x;
        }
        Ibus[r] = s;
        const double2 vr = V[r];
        const double2 sb = Sbus[r];
        double mr = vr.x * s.x + vr.y * s.y - sb.x;  // V * conj(I) - S
        const double mi = vr.y * s.x - vr.x * s.y - sb.y;
        if (P.distributed) mr += sa * P.w[r];
        Fbus[r] = make_double2(mr, mi);
        const int ip = P.xP[r], iq = P.xQ[r];
        if (ip >= 0) {
            x[ip] = (XT)mr;
            lmax = fmax(lmax, fabs(mr));
            lbad |= !isfinite(mr);
        }
        if (iq >= 0) {
            x[iq] = (XT)mi;
            lmax = fmax(lmax, fabs(mi));
            lbad |= !isfinite(mi);
        }
    }
    block_norm(S, lmax, lbad, norm, bad);
}

// dS/dVm and dS/dVa at V scattered into the LU array (and into Jout when requested).
template <typename LT>
__device__ void jacobian_fill(const DevPlan &P, Shared &S, const double2 *__restrict__ V,
                              const double2 *__restrict__ Ibus, LT *lu, double *Jout) {
    for (int p = threadIdx.x; p < P.nnzY; p += blockDim.x) {
        const int r = P.Rrow[p], c = P.Rj[p];
        double dvar, dvai;
        double2 dvm;
        dsbus(ybus_value(P, S, p), V[r], V[c], r == c, r == c ? Ibus[r] : make_double2(0.0, 0.0), dvar, dvai, dvm);
        const int4 t = P.ytarget[p];
        if (t.x >= 0) lu[t.x] = (LT)dvar;
        if (t.y >= 0) lu[t.y] = (LT)dvai;
        if (t.z >= 0) lu[t.z] = (LT)dvm.x;
        if (t.w >= 0) lu[t.w] = (LT)dvm.y;
        if (Jout) {
            const int4 j = P.yjpos[p];
            if (j.x >= 0) Jout[j.x] = dvar;
            if (j.y >= 0) Jout[j.y] = dvai;
            if (j.z >= 0) Jout[j.z] = dvm.x;
            if (j.w >= 0) Jout[j.w] = dvm.y;
        }
    }
    for (int i = threadIdx.x; i < P.nfill; i += blockDim.x) lu[P.fillpos[i]] = (LT)0;
    for (int i = threadIdx.x; i < P.nconst; i += blockDim.x) {
        lu[P.cpos[i]] = (LT)P.cval[i];
        if (Jout) Jout[P.cjpos[i]] = P.cval[i];
    }
}

// Right-looking refactorisation in conflict-free phases; sets S.piv_err on a zero pivot.
template <typename LT>
__device__ void refactor(const DevPlan &P, Shared &S, LT *lu) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int ph = 0; ph < P.nphases; ++ph) {
        const int4 Q = P.phases[ph];
        const int lanes = P.ph_lanes[ph];
        for (int e = Q.z + tid; e < Q.w; e += nt) {
            const int2 dv = P.divs[e];
            lu[dv.x] = lu[dv.x] / lu[dv.y];
        }
        const int per_warp = 32 / lanes;
        const int sub = lane & (lanes - 1);
        const int nslots = nw * per_warp;
        for (int g = Q.x + warp * per_warp + lane / lanes; g < Q.y; g += nslots) {
            const int4 G = P.grp[g];
            const int lc = P.grp_lc[g];
            const LT f = lu[G.y] / lu[G.z];  // U(c, j) / U(c, c)
            const int *d = P.dst + G.w;
            for (int s = sub; s < lc; s += lanes) lu[d[s]] -= lu[G.x + s] * f;
        }
        __syncthreads();
    }
    int zero = 0;
    for (int k = tid; k < P.m; k += nt) zero |= lu[P.dpos[k]] == (LT)0;
    if (zero) S.piv_err = 1;
    __syncthreads();
}

// Row-oriented, level-scheduled substitution.  upper == false: x_i -= L(i,:) x (unit
// diagonal); upper == true: x_i = (x_i - U(i,:) x) / U(i,i).
template <typename LT, typename XT, bool upper>
__device__ void tri_solve(const DevPlan &P, const LT *lu, XT *x) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int4 *desc = upper ? P.bwd_desc : P.fwd_desc;
    const int2 *pc = upper ? P.urow_pc : P.lrow_pc;
    const int4 *groups = upper ? P.bwd_groups : P.fwd_groups;
    const int ng = upper ? P.nbwd : P.nfwd;
    for (int g = 0; g < ng; ++g) {
        const int4 G = groups[g];
        if (G.z == 0) {
            const int lanes = G.w;
            const int per_warp = 32 / lanes;
            const int sub = lane & (lanes - 1);
            const int slot = lane / lanes;
            for (int base = G.x + warp * per_warp; base < G.y; base += nw * per_warp) {
                const int t = base + slot;
                XT s = (XT)0;
                int4 d = make_int4(-1, 0, 0, 0);
                if (t < G.y) {
                    d = desc[t];
                    for (int e = sub; e < d.z; e += lanes) {
                        const int2 q = pc[d.y + e];
                        s += (XT)lu[q.x] * x[q.y];
                    }
                }
                s = warp_sum(s, lanes);
                if (d.x >= 0 && sub == 0) {
                    if (upper) x[d.x] = (x[d.x] - s) / (XT)lu[d.w];
                    else x[d.x] -= s;
                }
            }
        } else if (warp == 0) {
            // chain: one row after the other; the next row's descriptor and first 32
            // entries are loaded while the current row is reduced
            int4 dn = desc[G.x];
            int2 qn = lane < dn.z ? pc[dn.y + lane] : make_int2(0, 0);
            for (int t = G.x; t < G.y; ++t) {
                const int4 d = dn;
                const int2 q = qn;
                if (t + 1 < G.y) {
                    dn = desc[t + 1];
                    qn = lane < dn.z ? pc[dn.y + lane] : make_int2(0, 0);
                }
                XT s = lane < d.z ? (XT)lu[q.x] * x[q.y] : (XT)0;
                for (int e = lane + 32; e < d.z; e += 32) {
                    const int2 q2 = pc[d.y + e];
                    s += (XT)lu[q2.x] * x[q2.y];
                }
                s = warp_sum(s, 32);
                if (lane == 0) {
                    if (upper) x[d.x] = (x[d.x] - s) / (XT)lu[d.w];
                    else x[d.x] -= s;
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
}

// FP64 residual of the Newton system, F - J dx, written as the next right-hand side.
// J dx is formed row by row from dS/dV (the FP64 Jacobian, never stored).
template <typename XT>
__device__ void newton_residual(const DevPlan &P, Shared &S, const double2 *__restrict__ V,
                                const double2 *__restrict__ Ibus, const double2 *__restrict__ Fbus,
                                const double *__restrict__ dxg, XT *x) {
    for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
        const int ip = P.xP[r], iq = P.xQ[r];
        if (ip < 0 && iq < 0) continue;
        const double2 vr = V[r];
        double accP = 0.0, accQ = 0.0;
        const int p1 = P.Rp[r + 1];
        for (int p = P.Rp[r]; p < p1; ++p) {
            const int c = P.Rj[p];
            const int ia = P.xVa[c], im = P.xVm[c];
            const double dA = ia >= 0 ? dxg[ia] : 0.0;
            const double dM = im >= 0 ? dxg[im] : 0.0;
            if (ia < 0 && im < 0) continue;
            double dvar, dvai;
            double2 dvm;
            dsbus(ybus_value(P, S, p), vr, V[c], r == c, r == c ? Ibus[r] : make_double2(0.0, 0.0), dvar, dvai,
                  dvm);
            accP += dvar * dA + dvm.x * dM;
            accQ += dvai * dA + dvm.y * dM;
        }
        if (P.distributed && ip >= 0) accP += P.wJ[r] * dxg[P.xSlack];
        const double2 F = Fbus[r];
        if (ip >= 0) x[ip] = (XT)(F.x - accP);
        if (iq >= 0) x[iq] = (XT)(F.y - accQ);
    }
}

template <typename LT, typename XT, bool LU_SMEM, bool REFINE>
__global__ void __launch_bounds__(512, 1) nr_batch_kernel(const DevPlan P, const BatchArgs A) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared S;
    const int tid = threadIdx.x;
    const int n = P.n, m = P.m;
    const size_t xbytes = ((size_t)m * sizeof(XT) + 15) & ~(size_t)15;
    XT *x = reinterpret_cast<XT *>(dyn);
    unsigned char *slab = A.scratch + (size_t)blockIdx.x * (size_t)A.slab_bytes;
    double2 *V = reinterpret_cast<double2 *>(slab);
    double2 *Ibus = V + n;
    double2 *Fbus = Ibus + n;
    double *Vm = reinterpret_cast<double *>(Fbus + n);
    double *Va = Vm + n;
    double *dxg = Va + n;
    const size_t bus_bytes = (((size_t)n * 64 + (size_t)m * 8) + 255) & ~(size_t)255;
    LT *lu = LU_SMEM ? reinterpret_cast<LT *>(dyn + xbytes) : reinterpret_cast<LT *>(slab + bus_bytes);

    for (;;) {
        if (tid == 0) S.job = atomicAdd(A.job_counter, 1);
        __syncthreads();
        const int job = S.job;
        __syncthreads();
        if (job >= A.njobs) break;
        const int first = A.job_first[job], count = A.job_count[job];
        for (int step = 0; step < count; ++step) {
            const int inst = first + step;
            const double2 *Sb = A.Sbus + (long long)inst * A.sbus_stride;
            if (step == 0 || !A.chain) {
                const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
                for (int b = tid; b < n; b += blockDim.x) {
                    const double2 v = v0[b];
                    V[b] = v;
                    Vm[b] = cabs2(v);
                    Va[b] = atan2(v.y, v.x);
                }
            } else {
                for (int b = tid; b < n; b += blockDim.x) {
                    const double2 v = V[b];
                    Vm[b] = cabs2(v);
                    Va[b] = atan2(v.y, v.x);
                }
            }
            if (tid == 0) {
                int k0 = 0, k1 = 0;
                if (A.ovr_ptr) {
                    k0 = A.ovr_ptr[inst];
                    k1 = A.ovr_ptr[inst + 1];
                }
                S.novr = min(k1 - k0, kMaxOverrides);
                S.piv_err = 0;
                S.slack_absorbed = 0.0;
            }
            __syncthreads();
            if (tid < S.novr) {
                const int k0 = A.ovr_ptr[inst];
                S.opos[tid] = A.ovr_pos[k0 + tid];
                S.oval[tid] = A.ovr_val[k0 + tid];
            }
            if (P.distributed) {
                double ls = 0.0;
                for (int b = tid; b < n; b += blockDim.x) ls += Sb[b].x;
                const double tot = block_sum(S, ls);
                if (tid == 0) S.slack_absorbed = tot;
            }
            __syncthreads();
            double norm;
            int bad;
            mismatch<XT>(P, S, V, Ibus, Fbus, Sb, x, norm, bad);
            bool conv = !bad && norm < A.tol;
            int it = 0, err = 0;
            double *Jout = (A.Jout && inst == A.j_inst) ? A.Jout : nullptr;
            while (!conv && it < A.max_iter) {
                ++it;
                jacobian_fill<LT>(P, S, V, Ibus, lu, Jout);
                __syncthreads();
                refactor<LT>(P, S, lu);
                if (S.piv_err) {
                    err = 6;  // SolverReFactor
                    break;
                }
                tri_solve<LT, XT, false>(P, lu, x);
                tri_solve<LT, XT, true>(P, lu, x);
                if (REFINE) {
                    for (int k = tid; k < m; k += blockDim.x) dxg[k] = (double)x[k];
                    __syncthreads();
                    newton_residual<XT>(P, S, V, Ibus, Fbus, dxg, x);
                    __syncthreads();
                    tri_solve<LT, XT, false>(P, lu, x);
                    tri_solve<LT, XT, true>(P, lu, x);
                }
                // voltage update
                double lmin = 1.0;
                for (int b = tid; b < n; b += blockDim.x) {
                    double vm, va;
                    if (P.distributed) {
                        vm = Vm[b];
                        va = Va[b];
                    } else {
                        const double2 v = V[b];
                        vm = cabs2(v);
                        va = atan2(v.y, v.x);
                    }
                    const int ia = P.xVa[b], im = P.xVm[b];
                    if (ia >= 0) va -= REFINE ? dxg[ia] + (double)x[ia] : (double)x[ia];
                    if (im >= 0) vm -= REFINE ? dxg[im] + (double)x[im] : (double)x[im];
                    double sn, cs;
                    sincos(va, &sn, &cs);
                    V[b] = make_double2(vm * cs, vm * sn);
                    Vm[b] = vm;
                    Va[b] = va;
                    lmin = fmin(lmin, vm);
                }
                if (P.distributed) {
                    const double dxs =
                        REFINE ? dxg[P.xSlack] + (double)x[P.xSlack] : (double)x[P.xSlack];
                    const double vmin = block_min(S, lmin);  // contains barriers
                    if (tid == 0) S.slack_absorbed -= dxs;
                    if (vmin < 0.0) {
                        for (int b = tid; b < n; b += blockDim.x) {
                            const double2 v = V[b];
                            Vm[b] = cabs2(v);
                            Va[b] = atan2(v.y, v.x);
                        }
                    }
                }
                __syncthreads();
                mismatch<XT>(P, S, V, Ibus, Fbus, Sb, x, norm, bad);
                if (bad) {
                    err = 3;  // InifiniteValue
                    break;
                }
                conv = norm < A.tol;
            }
            if (!conv && err == 0) err = 2;  // TooManyIterations
            double2 *vo = A.Vout + (long long)inst * n;
            for (int b = tid; b < n; b += blockDim.x) vo[b] = V[b];
            if (tid == 0) {
                A.iters[inst] = it;
                A.errs[inst] = err;
            }
            __syncthreads();
            if (A.chain && err != 0) {
                // the reference stops a time series at its first divergence
                for (int s2 = step + 1 + tid; s2 < count; s2 += blockDim.x) {
                    A.iters[first + s2] = 0;
                    A.errs[first + s2] = 8;  // NotInitError: not computed
                }
                break;
            }
        }
        __syncthreads();
    }
}

template <typename LT, typename XT, bool SM, bool RF>
cudaError_t launch_variant(const DevPlan &P, const BatchArgs &A, int threads, int grid, size_t smem,
                           cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(nr_batch_kernel<LT, XT, SM, RF>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    nr_batch_kernel<LT, XT, SM, RF><<<grid, threads, smem, st>>>(P, A);
    return cudaGetLastError();
}

template <typename LT, typename XT, bool SM, bool RF>
int occupancy_variant(int threads, size_t smem) {
    int nb = 0;
    if (cudaFuncSetAttribute(nr_batch_kernel<LT, XT, SM, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, nr_batch_kernel<LT, XT, SM, RF>, threads, smem) !=
        cudaSuccess)
        return 0;
    return nb;
}

}  // namespace

size_t slab_bytes(const DevPlan &P, int lu_bytes, bool lu_in_smem) {
    size_t bus = (((size_t)P.n * 64 + (size_t)P.m * 8) + 255) & ~(size_t)255;
    size_t lu = lu_in_smem ? 0 : (((size_t)P.nnzLU * lu_bytes + 255) & ~(size_t)255);
    return bus + lu;
}

size_t smem_bytes(const DevPlan &P, int lu_bytes, int x_bytes, bool lu_in_smem) {
    size_t xb = ((size_t)P.m * x_bytes + 15) & ~(size_t)15;
    return xb + (lu_in_smem ? (size_t)P.nnzLU * lu_bytes : 0);
}

cudaError_t launch_nr_batch(const DevPlan &P, const BatchArgs &A, int precision, int threads, int grid,
                            size_t smem, cudaStream_t stream) {
    const bool sm = A.lu_in_smem != 0;
    if (precision == 0) {
        return sm ? launch_variant<double, double, true, false>(P, A, threads, grid, smem, stream)
                  : launch_variant<double, double, false, false>(P, A, threads, grid, smem, stream);
    }
    if (A.refine)
        return sm ? launch_variant<float, float, true, true>(P, A, threads, grid, smem, stream)
                  : launch_variant<float, float, false, true>(P, A, threads, grid, smem, stream);
    return sm ? launch_variant<float, float, true, false>(P, A, threads, grid, smem, stream)
              : launch_variant<float, float, false, false>(P, A, threads, grid, smem, stream);
}

int nr_occupancy(int precision, bool lu_in_smem, bool refine, int threads, size_t smem) {
    if (precision == 0)
        return lu_in_smem ? occupancy_variant<double, double, true, false>(threads, smem)
                          : occupancy_variant<double, double, false, false>(threads, smem);
    if (refine)
        return lu_in_smem ? occupancy_variant<float, float, true, true>(threads, smem)
                          : occupancy_variant<float, float, false, true>(threads, smem);
    return lu_in_smem ? occupancy_variant<float, float, true, false>(threads, smem)
                      : occupancy_variant<float, float, false, false>(threads, smem);
}

}  // namespace l2g
