// Host construction of the spectral operators of one (ng, nz) grid.
//
// Follows Spectral::new (reference src/spectral/mod.rs:65-299): wavenumbers,
// hyperviscosity, dealiasing filter, semi-implicit operators, trapezoid weights,
// pressure Thomas factors (stored [kx + ng*ky + ng*ng*iz], iz < nz) and the
// compact d/dtheta factors.  Computed once in float64 and uploaded; the
// expressions keep the reference's operation order so that the uploaded
// operators match its own to the last bit where libm agrees.
#pragma once
#include <cmath>
#include <vector>

namespace sw {

struct SpectralHost {
    int ng = 0, nz = 0;
    std::vector<double> hlap, glap, rlap, helm, c2g2, simp, rope, fope, filt, diss, opak, rdis;
    std::vector<double> etdv, htdv, ap, etd1, htd1, theta, weight, hrkx, rk, spmf, alk;
    std::vector<int> kmag;
    int kmax = 0, kmaxred = 0;

    void build(int ng_, int nz_) {
        ng = ng_;
        nz = nz_;
        const size_t n2 = (size_t)ng * ng;
        const double pi = 3.14159265358979323846;
        const double cof = 4.0 * pi, cgw = 2.0 * pi, hbar = 0.4, cdamp = 10.0, nnu = 3.0;
        const double csq = cgw * cgw, fsq = cof * cof, gravity = csq / hbar;
        const double dt = 1.0 / (double)ng, dt2 = dt * (1.0 / 2.0), dt2i = 1.0 / dt2;
        const double dz = hbar / (double)nz, dzi = 1.0 / dz, dzisq = std::pow(dzi, 2.0);
        auto z2 = [&](std::vector<double>& v, size_t n) { v.assign(n, 0.0); };
        for (auto* v : {&hlap, &glap, &rlap, &helm, &c2g2, &simp, &rope, &fope, &filt, &diss, &opak, &rdis, &ap})
            z2(*v, n2);
        z2(etdv, n2 * nz); z2(htdv, n2 * nz);
        z2(etd1, nz); z2(htd1, nz); z2(theta, nz + 1); z2(weight, nz + 1);
        z2(hrkx, ng); z2(rk, ng); z2(spmf, ng + 1); z2(alk, ng);
        kmag.assign(n2, 0);
        // D2FFT::new wavenumbers (src/sta2dfft.rs:68-83), lx = 2 pi
        const double sc = pi / (2.0 * pi);
        for (int k = 1; k <= ng; k++) hrkx[k - 1] = sc * (double)k;
        rk[0] = 0.0;
        for (int k = 1; k < ng / 2; k++) rk[k] = rk[ng - k] = hrkx[2 * k - 1];
        rk[ng / 2] = hrkx[ng - 1];
        const double rkmax = (double)(ng / 2);
        kmax = (int)std::ceil(rkmax * std::sqrt(2.0));
        for (int ky = 0; ky < ng; ky++)
            for (int kx = 0; kx < ng; kx++) {
                int k = (int)std::round(std::sqrt(std::pow(rk[kx], 2.0) + std::pow(rk[ky], 2.0)));
                kmag[kx + (size_t)ng * ky] = k;
                spmf[k] += 1.0;
            }
        const double snorm = 4.0 * pi / (double)(ng * ng);
        spmf[0] = 0.0;
        for (int k = 1; k <= kmax; k++) {
            spmf[k] = snorm * (double)k / spmf[k];
            alk[k - 1] = std::log10((double)k);
        }
        kmaxred = ng / 2;
        const double anu = cdamp * cof / std::pow(rkmax, 2.0 * nnu);
        const double rkfsq = std::pow((double)ng / 3.0, 2.0);
        for (int ky = 0; ky < ng; ky++)
            for (int kx = 0; kx < ng; kx++) {
                const size_t i = kx + (size_t)ng * ky;
                const double rks = std::pow(rk[kx], 2.0) + std::pow(rk[ky], 2.0);
                hlap[i] = -rks;
                opak[i] = -(fsq + csq * rks);
                diss[i] = anu * std::pow(rks, nnu);
                if (rks > rkfsq) {
                    filt[i] = glap[i] = c2g2[i] = rlap[i] = helm[i] = rope[i] = rdis[i] = 0.0;
                } else {
                    filt[i] = 1.0;
                    glap[i] = gravity * rks;
                    c2g2[i] = -csq * rks;
                    rlap[i] = -1.0 / (rks + 1.0E-20);
                    helm[i] = 1.0 / opak[i];
                    rope[i] = c2g2[i] * helm[i];
                    rdis[i] = dt2i + diss[i];
                }
                const double rrsq = std::pow(dt2i + diss[i], 2.0);
                fope[i] = -c2g2[i] / (rrsq - opak[i]);
                simp[i] = 1.0 / (rrsq + fsq);
                diss[i] = 2.0 / (1.0 + dt2 * diss[i]);
            }
        rlap[0] = 0.0;
        for (int iz = 0; iz <= nz; iz++) {
            theta[iz] = dz * (double)iz;
            weight[iz] = 1.0;
        }
        weight[0] = 0.5;
        weight[nz] = 0.5;
        for (int iz = 0; iz <= nz; iz++) weight[iz] /= (double)nz;
        std::vector<double> a0(n2), a0b(n2), apb(n2);
        for (int ky = 0; ky < ng; ky++)
            for (int kx = 0; kx < ng; kx++) {
                const size_t i = kx + (size_t)ng * ky;
                const double rks = std::pow(rk[kx], 2.0) + std::pow(rk[ky], 2.0);
                a0[i] = -2.0 * dzisq - (5.0 / 6.0) * rks;
                a0b[i] = -dzisq - (1.0 / 3.0) * rks;
                ap[i] = dzisq - (1.0 / 12.0) * rks;
                apb[i] = dzisq - (1.0 / 6.0) * rks;
            }
        for (size_t i = 0; i < n2; i++) {
            htdv[i] = filt[i] / a0b[i];
            etdv[i] = -apb[i] * htdv[i];
        }
        for (int iz = 1; iz <= nz - 2; iz++)
            for (size_t i = 0; i < n2; i++) {
                htdv[i + n2 * iz] = filt[i] / (a0[i] + ap[i] * etdv[i + n2 * (iz - 1)]);
                etdv[i + n2 * iz] = -ap[i] * htdv[i + n2 * iz];
            }
        for (size_t i = 0; i < n2; i++)
            htdv[i + n2 * (nz - 1)] = filt[i] / (a0[i] + ap[i] * etdv[i + n2 * (nz - 2)]);
        htd1[0] = 1.0 / (2.0 / 3.0);
        etd1[0] = -(1.0 / 6.0) * htd1[0];
        for (int iz = 2; iz < nz; iz++) {
            htd1[iz - 1] = 1.0 / ((2.0 / 3.0) + (1.0 / 6.0) * etd1[iz - 2]);
            etd1[iz - 1] = -(1.0 / 6.0) * htd1[iz - 1];
        }
        htd1[nz - 1] = 1.0 / ((2.0 / 3.0) + (1.0 / 3.0) * etd1[nz - 2]);
    }

    const std::vector<double>* find(const std::string& name) const {
        if (name == "hlap") return &hlap;
        if (name == "glap") return &glap;
        if (name == "rlap") return &rlap;
        if (name == "helm") return &helm;
        if (name == "c2g2") return &c2g2;
        if (name == "simp") return &simp;
        if (name == "rope") return &rope;
        if (name == "fope") return &fope;
        if (name == "filt") return &filt;
        if (name == "diss") return &diss;
        if (name == "opak") return &opak;
        if (name == "rdis") return &rdis;
        if (name == "etdv") return &etdv;
        if (name == "htdv") return &htdv;
        if (name == "ap") return &ap;
        if (name == "etd1") return &etd1;
        if (name == "htd1") return &htd1;
        if (name == "theta") return &theta;
        if (name == "weight") return &weight;
        if (name == "hrkx" || name == "hrky") return &hrkx;
        if (name == "rk") return &rk;
        if (name == "spmf") return &spmf;
        if (name == "alk") return &alk;
        return nullptr;
    }
};

}  // namespace sw
