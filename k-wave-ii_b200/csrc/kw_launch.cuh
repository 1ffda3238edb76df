// kw_launch.cuh -- kernel launchers of one axis length.
//
// Each launcher picks the kernel of its length and tile width (full tiles of
// ks_lines(N) lines, half ones of ks_half(N) or narrow ones of ks_narrow(N)),
// sets its shared-memory limit and launches it on the plan's stream.  N = 0 selects the
// runtime-radix kernels of kw_kernels.cuh, which take any supported length.
// Included by kw_inst.cu only.
#pragma once

#include "kw_plan.cuh"
#include "kw_static.cuh"

namespace kw {
namespace launch {

template <int N, int TY>
kw_status ypass(kw_plan *P, bool inv, Spec4 bufs, dim3 grid, int kz0) {
    constexpr int NT = ks_threads(N, TY);
    constexpr size_t sh = (size_t)N * TY * sizeof(float2);
    if (inv) {
        KW_TRY(set_smem((const void *)ks_ypass<true, N, TY>, sh));
        ks_ypass<true, N, TY><<<grid, NT, sh, P->stream>>>(bufs, P->g, P->tw[1], kz0);
    } else {
        KW_TRY(set_smem((const void *)ks_ypass<false, N, TY>, sh));
        ks_ypass<false, N, TY><<<grid, NT, sh, P->stream>>>(bufs, P->g, P->tw[1], kz0);
    }
    return KW_OK;
}

template <int N, int TY>
kw_status ypass_fan(kw_plan *P, Spec4 bufs, dim3 grid, int kz0, const float2 *ddy, const float2 *ddz) {
    constexpr int NT = ks_threads(N, TY);
    constexpr size_t sh = (size_t)N * TY * sizeof(float2);
    KW_TRY(set_smem((const void *)ks_ypass_fan<N, TY>, sh));
    ks_ypass_fan<N, TY><<<grid, NT, sh, P->stream>>>(bufs, P->g, P->tw[1], kz0, ddy, ddz);
    return KW_OK;
}

template <int N, int NL>
kw_status xpass(kw_plan *P, Spec4 bufs, OpSet ops, int fanout, int kz0, int nkz, dim3 grid) {
    // fanout 2 is the 3-D gradient's (three outputs along x, y, z)
    if (fanout == 2) {
        if (!(ops.n == 3 && ops.axis[0] == 0 && ops.axis[1] == 1 && ops.axis[2] == 2))
            return fail(KW_ERR_INVALID, "internal: the gradient fan-out x-pass needs outputs along x, y and z");
        ks_xpass<N, NL, 2><<<grid, ks_threads(N, NL), 0, P->stream>>>(bufs, P->g, P->tw[0], P->op, ops, 2, kz0, nkz);
    } else if (fanout)
        ks_xpass<N, NL, 1><<<grid, ks_threads(N, NL), 0, P->stream>>>(bufs, P->g, P->tw[0], P->op, ops, fanout, kz0, nkz);
    else
        ks_xpass<N, NL, 0><<<grid, ks_threads(N, NL), 0, P->stream>>>(bufs, P->g, P->tw[0], P->op, ops, 0, kz0, nkz);
    return KW_OK;
}

template <int N, int PL>
kw_status zr2c(kw_plan *P, const float *R, float2 *H, dim3 grid) {
    constexpr size_t sh = (size_t)N * PL * sizeof(float2);
    KW_TRY(set_smem((const void *)ks_zr2c<N, PL>, sh));
    ks_zr2c<N, PL><<<grid, ks_threads(N, PL), sh, P->stream>>>(R, H, P->g, P->tw[2]);
    return KW_OK;
}

template <int N, int PL>
kw_status zc2r(kw_plan *P, const float2 *H, float *R, dim3 grid) {
    constexpr size_t sh = (size_t)N * PL * sizeof(float2);
    KW_TRY(set_smem((const void *)ks_zc2r<N, PL>, sh));
    ks_zc2r<N, PL><<<grid, ks_threads(N, PL), sh, P->stream>>>(H, R, P->g, P->tw[2]);
    return KW_OK;
}

template <int N, int PL>
kw_status stage_u(kw_plan *P, const StageU &a, dim3 grid) {
    using Z = ZStage<N, PL>;
    const size_t sh = (size_t)(Z::TILE + 2 * Z::SLICE) * sizeof(float2);
    StageUMaps m;
    bool tma = false;
    KW_TRY(stage_u_maps(P, a, Z::TX, &m, &tma));
    if constexpr (Z::TMA_OK) {
        if (tma) {
            // 128 bytes of slack for the kernel to align its TMA destinations
            KW_TRY(set_smem((const void *)ks_stage_u<N, PL, true>, sh + 128));
            ks_stage_u<N, PL, true><<<grid, Z::NT, sh + 128, P->stream>>>(a, P->tw[2], m);
            return KW_OK;
        }
    }
    KW_TRY(set_smem((const void *)ks_stage_u<N, PL, false>, sh));
    ks_stage_u<N, PL, false><<<grid, Z::NT, sh, P->stream>>>(a, P->tw[2], m);
    return KW_OK;
}

template <int N, int PL>
kw_status stage_r(kw_plan *P, const StageR &a, dim3 grid) {
    using Z = ZStage<N, PL>;
    const size_t sh = (size_t)(Z::TILE + 2 * Z::SLICE) * sizeof(float2);
    StageRMaps m;
    bool tma = false;
    KW_TRY(stage_r_maps(P, a, Z::TX, &m, &tma));
    // the spectrum rows come in boxes of at most 256 rows (tma_rows); the
    // TMA variant exists where every box starts 128-byte aligned
    if constexpr (Z::TMA_OK) {
        if (tma) {
            // 128 bytes of slack for the kernel to align its TMA destinations
            KW_TRY(set_smem((const void *)ks_stage_r<N, PL, true>, sh + 128));
            ks_stage_r<N, PL, true><<<grid, Z::NT, sh + 128, P->stream>>>(a, P->tw[2], m);
            return KW_OK;
        }
    }
    {
        KW_TRY(set_smem((const void *)ks_stage_r<N, PL, false>, sh));
        ks_stage_r<N, PL, false><<<grid, Z::NT, sh, P->stream>>>(a, P->tw[2], m);
    }
    return KW_OK;
}

template <int N, int PL>
kw_status stage_p(kw_plan *P, const StageP &a, dim3 grid) {
    using Z = ZStage<N, PL>;
    const size_t sh = (size_t)(Z::TILE + 2 * Z::SLICE) * sizeof(float2);
    StagePMaps m;
    bool tma = false;
    KW_TRY(stage_p_maps(P, a, Z::TX, &m, &tma));
    if constexpr (Z::TMA_OK) {
        if (tma) {
            // 128 bytes of slack for the kernel to align its TMA destinations
            KW_TRY(set_smem((const void *)ks_stage_p<N, PL, true>, sh + 128));
            ks_stage_p<N, PL, true><<<grid, Z::NT, sh + 128, P->stream>>>(a, P->tw[2], m);
            return KW_OK;
        }
    }
    KW_TRY(set_smem((const void *)ks_stage_p<N, PL, false>, sh));
    ks_stage_p<N, PL, false><<<grid, Z::NT, sh, P->stream>>>(a, P->tw[2], m);
    return KW_OK;
}

}  // namespace launch

template <int N>
kw_status YLaunch<N>::run(kw_plan *P, bool inv, Spec4 bufs, int nf, int kz0, int nkz) {
    dim3 grid((P->g.N0 + P->TY - 1) / P->TY, N > 0 ? nkz : P->g.N2h, nf);
    if constexpr (N > 0) {
        if (P->TY == ks_lines(N)) KW_TRY((launch::ypass<N, ks_lines(N)>(P, inv, bufs, grid, kz0)));
        else if (P->TY == ks_half(N)) KW_TRY((launch::ypass<N, ks_half(N)>(P, inv, bufs, grid, kz0)));
        else KW_TRY((launch::ypass<N, ks_narrow(N)>(P, inv, bufs, grid, kz0)));
    } else {
        size_t sh = (size_t)P->TY * P->g.N1 * sizeof(float2);
        if (inv) {
            KW_TRY(set_smem((const void *)k_ypass<true, 0, 0>, sh));
            k_ypass<true, 0, 0><<<grid, kThreads, sh, P->stream>>>(bufs, P->g, P->fft[1], P->TY);
        } else {
            KW_TRY(set_smem((const void *)k_ypass<false, 0, 0>, sh));
            k_ypass<false, 0, 0><<<grid, kThreads, sh, P->stream>>>(bufs, P->g, P->fft[1], P->TY);
        }
    }
    return launched(P);
}

template <int N>
kw_status YLaunch<N>::run_fan(kw_plan *P, Spec4 bufs, int kz0, int nkz, const float2 *ddy, const float2 *ddz) {
    if constexpr (N > 0) {
        dim3 grid((P->g.N0 + P->TY - 1) / P->TY, nkz, 2);
        if (P->TY == ks_lines(N)) KW_TRY((launch::ypass_fan<N, ks_lines(N)>(P, bufs, grid, kz0, ddy, ddz)));
        else if (P->TY == ks_half(N)) KW_TRY((launch::ypass_fan<N, ks_half(N)>(P, bufs, grid, kz0, ddy, ddz)));
        else KW_TRY((launch::ypass_fan<N, ks_narrow(N)>(P, bufs, grid, kz0, ddy, ddz)));
        return launched(P);
    } else {
        return fail(KW_ERR_INVALID, "internal: the gradient fan-out y-pass needs a compile-time axis length");
    }
}

template <int N>
kw_status XLaunch<N>::run(kw_plan *P, Spec4 bufs, OpSet ops, int fanout, int nf, int kz0, int nkz) {
    const int lines = P->g.N1 * (N > 0 ? nkz : P->g.N2h);
    dim3 grid((lines + P->NL - 1) / P->NL, 1, fanout ? 1 : nf);
    if constexpr (N > 0) {
        if (P->NL == ks_xlines(N)) KW_TRY((launch::xpass<N, ks_xlines(N)>(P, bufs, ops, fanout, kz0, nkz, grid)));
        else if (P->NL == ks_xhalf(N)) KW_TRY((launch::xpass<N, ks_xhalf(N)>(P, bufs, ops, fanout, kz0, nkz, grid)));
        else KW_TRY((launch::xpass<N, ks_xnarrow(N)>(P, bufs, ops, fanout, kz0, nkz, grid)));
    } else {
        size_t sh = (size_t)(fanout ? 2 : 1) * P->NL * P->g.N0 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_xpass<0, 0>, sh));
        k_xpass<0, 0><<<grid, kThreads, sh, P->stream>>>(bufs, P->g, P->fft[0], P->NL, P->op, ops, fanout);
    }
    return launched(P);
}

template <int N>
kw_status ZR2CLaunch<N>::run(kw_plan *P, const float *R, float2 *H) {
    dim3 grid((P->g.N0 + 2 * P->PL_z - 1) / (2 * P->PL_z), P->g.N1, 1);
    if constexpr (N > 0) {
        if (P->PL_z == ks_lines(N)) KW_TRY((launch::zr2c<N, ks_lines(N)>(P, R, H, grid)));
        else if (P->PL_z == ks_half(N)) KW_TRY((launch::zr2c<N, ks_half(N)>(P, R, H, grid)));
        else KW_TRY((launch::zr2c<N, ks_narrow(N)>(P, R, H, grid)));
    } else {
        size_t sh = (size_t)P->PL_z * P->g.N2 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_zr2c<0, 0>, sh));
        k_zr2c<0, 0><<<grid, kThreads, sh, P->stream>>>(R, H, P->g, P->fft[2], P->PL_z);
    }
    return launched(P);
}

template <int N>
kw_status ZC2RLaunch<N>::run(kw_plan *P, const float2 *H, float *R) {
    dim3 grid((P->g.N0 + 2 * P->PL_z - 1) / (2 * P->PL_z), P->g.N1, 1);
    if constexpr (N > 0) {
        if (P->PL_z == ks_lines(N)) KW_TRY((launch::zc2r<N, ks_lines(N)>(P, H, R, grid)));
        else if (P->PL_z == ks_half(N)) KW_TRY((launch::zc2r<N, ks_half(N)>(P, H, R, grid)));
        else KW_TRY((launch::zc2r<N, ks_narrow(N)>(P, H, R, grid)));
    } else {
        size_t sh = (size_t)P->PL_z * P->g.N2 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_zc2r<0, 0>, sh));
        k_zc2r<0, 0><<<grid, kThreads, sh, P->stream>>>(H, R, P->g, P->fft[2], P->PL_z);
    }
    return launched(P);
}

template <int N>
kw_status ULaunch<N>::run(kw_plan *P, StageU a) {
    dim3 grid((P->g.N0 + 2 * a.PL - 1) / (2 * a.PL), P->g.N1, P->D);
    if constexpr (N > 0) {
        if (a.PL == ks_lines(N)) KW_TRY((launch::stage_u<N, ks_lines(N)>(P, a, grid)));
        else if (a.PL == ks_half(N)) KW_TRY((launch::stage_u<N, ks_half(N)>(P, a, grid)));
        else KW_TRY((launch::stage_u<N, ks_narrow(N)>(P, a, grid)));
    } else {
        size_t sh = (size_t)a.PL * P->g.N2 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_stage_u<0, 0>, sh));
        k_stage_u<0, 0><<<grid, kThreads, sh, P->stream>>>(a);
    }
    return launched(P);
}

template <int N>
kw_status RLaunch<N>::run(kw_plan *P, StageR a) {
    dim3 grid((P->g.N0 + 2 * a.PL - 1) / (2 * a.PL), P->g.N1, 1);
    if constexpr (N > 0) {
        if (a.PL == ks_lines(N)) KW_TRY((launch::stage_r<N, ks_lines(N)>(P, a, grid)));
        else if (a.PL == ks_half(N)) KW_TRY((launch::stage_r<N, ks_half(N)>(P, a, grid)));
        else KW_TRY((launch::stage_r<N, ks_narrow(N)>(P, a, grid)));
    } else {
        size_t sh = (size_t)4 * a.PL * P->g.N2 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_stage_r<0, 0>, sh));
        k_stage_r<0, 0><<<grid, kThreads, sh, P->stream>>>(a);
    }
    return launched(P);
}

template <int N>
kw_status PLaunch<N>::run(kw_plan *P, StageP a) {
    dim3 grid((P->g.N0 + 2 * a.PL - 1) / (2 * a.PL), P->g.N1, 1);
    if constexpr (N > 0) {
        if (a.PL == ks_lines(N)) KW_TRY((launch::stage_p<N, ks_lines(N)>(P, a, grid)));
        else if (a.PL == ks_half(N)) KW_TRY((launch::stage_p<N, ks_half(N)>(P, a, grid)));
        else KW_TRY((launch::stage_p<N, ks_narrow(N)>(P, a, grid)));
    } else {
        size_t sh = (size_t)2 * a.PL * P->g.N2 * sizeof(float2);
        KW_TRY(set_smem((const void *)k_stage_p<0, 0>, sh));
        k_stage_p<0, 0><<<grid, kThreads, sh, P->stream>>>(a);
    }
    return launched(P);
}

}  // namespace kw
