// Warp-per-site SOAP kernels (forward expansion + power spectrum, adjoint back-scatter).
// Included by soap.cu inside namespace tgap (shares the harmonic constants in constant memory).
//
// A warp owns one central site. The site's in-cutoff pairs are compacted with a ballot into
// groups of at most 32; each lane then evaluates one pair completely (radial quadrature, Bessel
// ratios, every real harmonic) with l_max fixed at compile time, so all harmonic indices and
// per-l factors resolve to registers and every lane walks the same (l, m) sequence (shared-
// memory reads of per-site data are broadcasts). Four warps share a CTA; nothing synchronizes
// across warps. Pair and atom indices are bounds-checked: a failed check is recorded in the
// device check word and the access is skipped.
#pragma once

constexpr int kWarpsPerCta = 4;

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// f_l = i_l(k)/i_0(k), l = 0..L+1, same rule as bessel_ratios, unrolled for a fixed L.
template <class T, int L>
__device__ __forceinline__ void bessel_ratios_fixed(T k, T f[L + 2])
{
    if (k < (T)1.0e-12) {
#pragma unroll
        for (int l = 0; l <= L + 1; ++l) f[l] = (l == 0) ? (T)1 : (T)0;
        return;
    }
    if (k > (T)(L + 2)) {
        f[0] = 1;
        f[1] = t_tanh_inv<T>(k) - (T)1 / k;
#pragma unroll
        for (int l = 1; l <= L; ++l) f[l + 1] = f[l - 1] - (T)(2 * l + 1) / k * f[l];
    } else {
        T rho = 0;
        for (int l = L + 1 + 32; l > L + 1; --l) rho = k / ((T)(2 * l + 1) + k * rho);
        T ratio[L + 2];
#pragma unroll
        for (int l = L + 1; l >= 1; --l) {
            rho = k / ((T)(2 * l + 1) + k * rho);
            ratio[l] = rho;
        }
        f[0] = 1;
#pragma unroll
        for (int l = 1; l <= L + 1; ++l) f[l] = f[l - 1] * ratio[l];
    }
}

// Every real harmonic of u for a fixed L: fn(k, l, Y, dY/dux, dY/duy, dY/duz), k = l^2 + ...
template <class T, int L, bool GRAD, class F>
__device__ __forceinline__ void ylm_all(T ux, T uy, T uz, F &&fn)
{
    T Cc = 1, Sc = 0, Cp = 0, Sp = 0;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
        if (m > 0) {
            Cp = Cc;
            Sp = Sc;
            const T cn = ux * Cc - uy * Sc;
            const T sn = ux * Sc + uy * Cc;
            Cc = cn;
            Sc = sn;
        }
        T Q2 = 0, Q1 = 0, dQ2 = 0, dQ1 = 0;
        const T qmm = (T)c_ylm.dfact[m];
#pragma unroll
        for (int l = m; l <= L; ++l) {
            T Q, dQ;
            if (l == m) {
                Q = qmm;
                dQ = 0;
            } else if (l == m + 1) {
                Q = (T)(2 * m + 1) * uz * qmm;
                dQ = (T)(2 * m + 1) * qmm;
            } else {
                const T inv = (T)(1.0 / (double)(l - m));
                Q = ((T)(2 * l - 1) * uz * Q1 - (T)(l + m - 1) * Q2) * inv;
                dQ = ((T)(2 * l - 1) * (Q1 + uz * dQ1) - (T)(l + m - 1) * dQ2) * inv;
            }
            Q2 = Q1;
            Q1 = Q;
            dQ2 = dQ1;
            dQ1 = dQ;
            const T N = (T)c_ylm.norm[l * (l + 1) / 2 + m];
            if (m == 0) {
                fn(l * l, l, N * Q, (T)0, (T)0, GRAD ? N * dQ : (T)0);
            } else {
                const T NQ = N * Q;
                if (GRAD) {
                    const T NQm = NQ * (T)m;
                    fn(l * l + 2 * m - 1, l, NQ * Cc, NQm * Cp, -NQm * Sp, N * dQ * Cc);
                    fn(l * l + 2 * m, l, NQ * Sc, NQm * Sp, NQm * Cp, N * dQ * Sc);
                } else {
                    fn(l * l + 2 * m - 1, l, NQ * Cc, (T)0, (T)0, (T)0);
                    fn(l * l + 2 * m, l, NQ * Sc, (T)0, (T)0, (T)0);
                }
            }
        }
    }
}

// Pair acceptance used by the compaction: species channel known and 0 < r < rcut_hard(s).
__device__ __forceinline__ bool pair_in_cutoff(const SoapParams &P, int64_t k, const double *__restrict__ rjs,
                                               const int *__restrict__ nsp)
{
    const int s = nsp[k] - 1;
    if (s < 0 || s >= P.n_species) return false;
    const double r = rjs[k];
    return r > 0.0 && r < P.rcut_hard[s];
}

// Compacts the next (at most 32) in-cutoff pairs of [scan, ke) into idx[]; returns the count
// and advances scan past the last pair taken.
__device__ __forceinline__ int compact_pairs(const SoapParams &P, int64_t &scan, int64_t ke,
                                             const double *__restrict__ rjs, const int *__restrict__ nsp,
                                             long long *idx, int lane)
{
    int cnt = 0;
    while (cnt < 32 && scan < ke) {
        const int64_t k = scan + lane;
        const bool ok = k < ke && pair_in_cutoff(P, k, rjs, nsp);
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        const int nv = __popc(mask);
        const int room = 32 - cnt;
        const int rank = __popc(mask & lanemask_lt());
        if (ok && rank < room) idx[cnt + rank] = (long long)k;
        if (nv > room) {
            // resume at the first in-cutoff pair that did not fit
            scan += __fns(mask, 0, room + 1);
            cnt = 32;
            break;
        }
        cnt += nv;
        scan += 32;
    }
    __syncwarp();
    return cnt;
}

// Radial coefficients (and optionally d/dr) of one pair evaluated by one lane.
template <class T, bool DERIV>
__device__ __forceinline__ void radial_lane(const SoapParams &P, int s, T r, const T *__restrict__ xq,
                                            const T *__restrict__ tq, T R[kMaxAlpha], T dR[kMaxAlpha])
{
    const int am = P.alpha_max[s];
    const T rc = (T)P.rcut_hard[s];
    const T x = r / rc;
    const T sig = ((T)P.sigma_r[s] + (T)P.sigma_r_scaling[s] * r) / rc;
    const T dsig = (T)P.sigma_r_scaling[s];
    T A, dA;
    radial_amplitude<T>(P, s, x, sig, dsig, &A, &dA);
    T sum[kMaxAlpha], dsum[kMaxAlpha];
#pragma unroll
    for (int n = 0; n < kMaxAlpha; ++n) {
        sum[n] = 0;
        dsum[n] = 0;
    }
    const T inv2s2 = (T)1 / ((T)2 * sig * sig);
    const T is2 = (T)2 * inv2s2;
    const T ds3 = dsig * is2 / sig;
    const T *xs = xq + P.node_off[s];
    const T *ts = tq + P.tq_off[s];
    const int nn = P.n_nodes[s];
    for (int q = 0; q < nn; ++q) {
        const T u = xs[q] - x;
        const T G = t_exp<T>(-u * u * inv2s2);
        const T *t = ts + q * am;
        const T dG = DERIV ? G * (u * is2 + u * u * ds3) : (T)0;
#pragma unroll
        for (int n = 0; n < kMaxAlpha; ++n) {
            if (n < am) {
                sum[n] += t[n] * G;
                if (DERIV) dsum[n] += t[n] * dG;
            }
        }
    }
    const T gs = (T)P.global_scaling[s];
#pragma unroll
    for (int n = 0; n < kMaxAlpha; ++n) {
        R[n] = gs * A * sum[n];
        if (DERIV) dR[n] = gs * (dA * sum[n] + A * dsum[n]) / rc;
    }
}

// ----------------------------------------------------------------------------- forward

template <class T, int L, bool SPLIT>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_soap_fwd_warp(
    SoapParams P, const T *__restrict__ xq, const T *__restrict__ tq, const T *__restrict__ central,
    const int *__restrict__ sites, int n_rows, const int64_t *__restrict__ start,
    const double *__restrict__ rjs, const double *__restrict__ xyz, const int *__restrict__ nsp,
    T *__restrict__ c_out, T *__restrict__ q_out, int q_ld, T *__restrict__ norm_out,
    __nv_bfloat16 *__restrict__ q_hi, __nv_bfloat16 *__restrict__ q_lo, int warp_smem, int *check)
{
    constexpr int NLM = (L + 1) * (L + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * kWarpsPerCta + warp;
    if (row >= n_rows) return;
    unsigned char *wbase = smem_raw + (size_t)warp * warp_smem;
    const int nmax = P.n_max, dim = P.dim, nout = nmax * NLM;
    long long *idx = reinterpret_cast<long long *>(wbase);  // [32] compacted pair indices
    T *Rs = reinterpret_cast<T *>(wbase + 256);             // [32][nmax]
    T *As = Rs + 32 * nmax;                                 // [32][NLM]   (reused for p)
    T *cs = As + (32 * NLM > dim ? 32 * NLM : dim);         // [nmax][NLM]

    const int site = sites ? sites[row] : row;
    const int64_t kb = start[site], ke = start[site + 1];
    int64_t scan = kb + 1;
    bool first = true;
    do {
        const int cnt = compact_pairs(P, scan, ke, rjs, nsp, idx, lane);
        if (cnt == 0 && !first) break;
        if (lane < cnt) {
            const int64_t k = idx[lane];
            const bool in_site = k > kb && k < ke;
            if (!in_site) check_fail(check, kCheckFwdPair, k, site);
            const int s = in_site ? nsp[k] - 1 : 0;
            const T r = in_site ? (T)rjs[k] : (T)1;
            const T ir = (T)1 / r;
            const T ux = in_site ? (T)xyz[3 * k] * ir : (T)0, uy = in_site ? (T)xyz[3 * k + 1] * ir : (T)0,
                    uz = in_site ? (T)xyz[3 * k + 2] * ir : (T)1;
            T R[kMaxAlpha], dR[kMaxAlpha];
            radial_lane<T, false>(P, s, r, xq, tq, R, dR);
            T *Rrow = Rs + lane * nmax;
            for (int n = 0; n < nmax; ++n) Rrow[n] = 0;
            const int off = P.n_off[s], am = P.alpha_max[s];
#pragma unroll
            for (int n = 0; n < kMaxAlpha; ++n)
                if (n < am && in_site) Rrow[off + n] = R[n];
            const T st = (T)P.sigma_t[s] + (T)P.sigma_t_scaling[s] * r;
            T f[L + 2];
            bessel_ratios_fixed<T, L>(r * r / (st * st), f);
            T *Arow = As + lane * NLM;
            ylm_all<T, L, false>(ux, uy, uz, [&](int kk, int l, T Y, T, T, T) { Arow[kk] = f[l] * Y; });
        }
        __syncwarp();
        for (int o = lane; o < nout; o += 32) {
            const int n = o / NLM, kk = o - n * NLM;
            T acc = first ? (T)0 : cs[o];
            for (int p = 0; p < cnt; ++p) acc += Rs[p * nmax + n] * As[p * NLM + kk];
            cs[o] = acc;
        }
        __syncwarp();
        first = false;
    } while (scan < ke);

    // central atom on l = 0 of its own species block
    const int s_self = nsp[kb] - 1;
    if (s_self >= 0 && s_self < P.n_species)
        for (int n = lane; n < P.alpha_max[s_self]; n += 32)
            cs[(P.n_off[s_self] + n) * NLM] += central[P.n_off[s_self] + n];
    __syncwarp();
    for (int o = lane; o < nout; o += 32) c_out[(size_t)row * nout + o] = cs[o];
    // power spectrum into the (free) A area
    T *ps = As;
    T part = 0;
    for (int d = lane; d < dim; d += 32) {
        int n, np, l;
        ps_decode(d, nmax, L, &n, &np, &l);
        const T *a = cs + n * NLM, *b = cs + np * NLM;
        T acc = 0;
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) acc += a[kk] * b[kk];
        const T v = (n == np) ? acc : acc * (T)1.4142135623730951;
        ps[d] = v;
        part += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const T nrm = t_sqrt<T>(part);
    const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
    __syncwarp();
    for (int d = lane; d < q_ld; d += 32) {
        const T qv = d < dim ? ps[d] * inv : (T)0;
        q_out[(size_t)row * q_ld + d] = qv;
        if (SPLIT) {
            const float qf = (float)qv;
            const __nv_bfloat16 h = __float2bfloat16_rn(qf);
            q_hi[(size_t)row * q_ld + d] = h;
            q_lo[(size_t)row * q_ld + d] = __float2bfloat16_rn(qf - __bfloat162float(h));
        }
    }
    if (lane == 0) norm_out[row] = nrm;
}

// ----------------------------------------------------------------------------- adjoint

// g = dE/dq per row. Pair forces go to forces[3 * jatom] with FP64 atomics, the site's own
// force (minus the sum) to forces[3 * jatom[self]], and the row's virial (xx yy zz xy xz yz)
// to vir_rows[6 * row] for a later per-structure reduction.
template <class T, class GT, int L>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_soap_bwd_warp(
    SoapParams P, const T *__restrict__ xq, const T *__restrict__ tq, const int *__restrict__ sites,
    int n_rows, const int64_t *__restrict__ start, const double *__restrict__ rjs,
    const double *__restrict__ xyz, const int *__restrict__ nsp, const int *__restrict__ jatom,
    const T *__restrict__ c_in, const T *__restrict__ q_in, int q_ld, const T *__restrict__ norm_in,
    const GT *__restrict__ g_in, int g_ld, double *__restrict__ forces, double *__restrict__ vir_rows,
    int warp_smem, int n_atoms, int *check)
{
    constexpr int NLM = (L + 1) * (L + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = blockIdx.x * kWarpsPerCta + warp;
    if (row >= n_rows) return;
    unsigned char *wbase = smem_raw + (size_t)warp * warp_smem;
    const int nmax = P.n_max, dim = P.dim, nout = nmax * NLM;
    long long *idx = reinterpret_cast<long long *>(wbase);  // [32] compacted pair indices
    T *cs = reinterpret_cast<T *>(wbase + 256);             // [nmax][NLM]
    T *Gc = cs + nout;                                      // [nmax][NLM]
    T *hs = Gc + nout;                                      // [dim]

    const int site = sites ? sites[row] : row;
    const int64_t kb = start[site], ke = start[site + 1];
    for (int o = lane; o < nout; o += 32) cs[o] = c_in[(size_t)row * nout + o];
    T qg = 0;
    for (int d = lane; d < dim; d += 32) qg += q_in[(size_t)row * q_ld + d] * (T)g_in[(size_t)row * g_ld + d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qg += __shfl_xor_sync(0xffffffffu, qg, o);
    const T nrm = norm_in[row];
    const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
    for (int d = lane; d < dim; d += 32)
        hs[d] = ((T)g_in[(size_t)row * g_ld + d] - q_in[(size_t)row * q_ld + d] * qg) * inv;
    __syncwarp();
    // dE/dc_{n,lm} = sum_n' M_l[n][n'] c_{n',lm}
    for (int o = lane; o < nout; o += 32) {
        const int n = o / NLM, kk = o - n * NLM;
        int l = 0;
        while ((l + 1) * (l + 1) <= kk) ++l;
        T acc = 0;
        for (int np = 0; np < nmax; ++np) {
            const T h = hs[ps_index(n, np, nmax, L, l)];
            acc += ((np == n) ? (T)2 * h : (T)1.4142135623730951 * h) * cs[np * NLM + kk];
        }
        Gc[o] = acc;
    }
    __syncwarp();

    double fs0 = 0, fs1 = 0, fs2 = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    int64_t scan = kb + 1;
    while (scan < ke) {
        const int cnt = compact_pairs(P, scan, ke, rjs, nsp, idx, lane);
        if (cnt == 0) break;
        const bool mine = lane < cnt;
        const int64_t k = mine ? idx[lane] : kb;
        const bool in_site = k > kb && k < ke;
        if (mine && !in_site) check_fail(check, kCheckBwdPair, k, site);
        if (mine && in_site) {
            const int s = nsp[k] - 1;
            const double xd0 = xyz[3 * k], xd1 = xyz[3 * k + 1], xd2 = xyz[3 * k + 2];
            const T r = (T)rjs[k];
            const T ir = (T)1 / r;
            const T u0 = (T)xd0 * ir, u1 = (T)xd1 * ir, u2 = (T)xd2 * ir;
            T R[kMaxAlpha], dR[kMaxAlpha];
            radial_lane<T, true>(P, s, r, xq, tq, R, dR);
            const T st = (T)P.sigma_t[s] + (T)P.sigma_t_scaling[s] * r;
            const T kap = r * r / (st * st);
            const T dkap = (T)2 * r / (st * st) - (T)2 * r * r * (T)P.sigma_t_scaling[s] / (st * st * st);
            T f[L + 2];
            bessel_ratios_fixed<T, L>(kap, f);
            const T ikap = kap > (T)0 ? (T)1 / kap : (T)0;
            const int off = P.n_off[s], am = P.alpha_max[s];
            const T *G = Gc + off * NLM;
            T w0 = 0, w1 = 0, w2 = 0;
            ylm_all<T, L, true>(u0, u1, u2, [&](int kk, int l, T Y, T gx, T gy, T gz) {
                T U = 0, V = 0;
#pragma unroll
                for (int n = 0; n < kMaxAlpha; ++n) {
                    if (n < am) {
                        const T gv = G[n * NLM + kk];
                        U += gv * R[n];
                        V += gv * dR[n];
                    }
                }
                const T fl = f[l];
                const T dfl = (f[l + 1] + (T)l * ikap * fl - fl * f[1]) * dkap;
                const T ug = u0 * gx + u1 * gy + u2 * gz;
                const T radial_part = fl * Y * V + U * dfl * Y;
                const T tang = U * fl * ir;
                w0 += u0 * radial_part + tang * (gx - u0 * ug);
                w1 += u1 * radial_part + tang * (gy - u1 * ug);
                w2 += u2 * radial_part + tang * (gz - u2 * ug);
            });
            // w = dE_i/dr_ij: force -w on the neighbor, +w on the site (its self slot)
            const double f0 = -(double)w0, f1 = -(double)w1, f2 = -(double)w2;
            const int j = jatom[k];
            if (j >= 0 && j < n_atoms) {
                atomicAdd(forces + 3 * (size_t)j, f0);
                atomicAdd(forces + 3 * (size_t)j + 1, f1);
                atomicAdd(forces + 3 * (size_t)j + 2, f2);
            } else {
                check_fail(check, kCheckBwdAtom, k, j);
            }
            fs0 -= f0;
            fs1 -= f1;
            fs2 -= f2;
            v0 += f0 * xd0;
            v1 += f1 * xd1;
            v2 += f2 * xd2;
            v3 += 0.5 * (f0 * xd1 + f1 * xd0);
            v4 += 0.5 * (f0 * xd2 + f2 * xd0);
            v5 += 0.5 * (f1 * xd2 + f2 * xd1);
        }
        __syncwarp();
    }
    double vals[9] = {fs0, fs1, fs2, v0, v1, v2, v3, v4, v5};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vals[i] += __shfl_xor_sync(0xffffffffu, vals[i], o);
    }
    if (lane < 3) {
        const double fv = lane == 0 ? vals[0] : (lane == 1 ? vals[1] : vals[2]);
        const int js = jatom[kb];
        if (js >= 0 && js < n_atoms)
            atomicAdd(forces + 3 * (size_t)js + lane, fv);
        else if (lane == 0)
            check_fail(check, kCheckSelfAtom, kb, js);
    }
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < 6; ++c) vir_rows[6 * (size_t)row + c] = vals[3 + c];
    }
}

// Sum of the row virials of each structure (rows of one structure are contiguous because sites
// ascend); adds into virial[9 * b] (column-major 3x3, symmetric). One CTA per structure.
__global__ void k_virial_reduce(int n_rows, const int *__restrict__ sites, const int *__restrict__ struct_off,
                                const double *__restrict__ vir_rows, double *__restrict__ virial)
{
    const int b = blockIdx.x;
    // no offsets: one structure holding every row
    const int a0 = struct_off ? struct_off[b] : INT_MIN, a1 = struct_off ? struct_off[b + 1] : INT_MAX;
    auto lower = [&](int a) {
        int lo = 0, hi = n_rows;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const int sv = sites ? sites[mid] : mid;
            if (sv < a)
                lo = mid + 1;
            else
                hi = mid;
        }
        return lo;
    };
    const int r0 = lower(a0), r1 = lower(a1);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[c] += vir_rows[6 * (size_t)r + c];
    __shared__ double red[6][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[threadIdx.x][i];
        const int ix[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        const int a = ix[threadIdx.x][0], c = ix[threadIdx.x][1];
        double *V = virial + 9 * (size_t)b;
        V[a + 3 * c] += v;
        if (a != c) V[c + 3 * a] += v;
    }
}
