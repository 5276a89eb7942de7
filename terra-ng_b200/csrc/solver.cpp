// Solver layer: multigrid hierarchy, Chebyshev-Jacobi smoothing, coarsest CG,
// block-triangular preconditioner and FGMRES (see tn_solver.hpp).
//
// Host code only orchestrates: every vector operation is a device kernel, and
// scalars that the next kernel needs (Gram-Schmidt coefficients, norms) stay in
// device memory. FGMRES waits for the device once per iteration, to read the
// new Hessenberg column for the Givens rotations and the convergence test
// (the reference waits at every dot product).
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>

#include "tn_solver.hpp"

namespace tn {

namespace {
int64_t pad64(int64_t n) { return (n + 63) / 64 * 64; }
void    chk(int rc, const char* what)
{
    if (rc != 0) throw Error(kErrCuda, std::string(what) + " launch failed");
}
template <typename T>
void lin(int64_t n, T* y, T c0, int nt, const T* c, const T* x0, const T* x1, cudaStream_t st)
{
    T*       yy[1] = {y};
    const T* a[1]  = {x0};
    const T* b[1]  = {x1};
    chk(lincomb<T>(n, 1, yy, c0, nt, c, a, b, nullptr, st), "lincomb");
}
}  // namespace

VecDesc velocity_desc(const DeviceLevel& L)
{
    VecDesc d;
    d.nseg         = 1;
    d.seg[0].n     = L.nodes();
    d.seg[0].stride = pad64(L.nodes());
    d.seg[0].ncomp = 3;
    d.seg[0].nr    = L.nr();
    d.seg[0].owned = L.owned_lat.as<uint8_t>();
    d.seg[0].rdiv  = reciprocal_nr(L.nr());
    d.total        = 3 * d.seg[0].stride;
    return d;
}

VecDesc scalar_desc(const DeviceLevel& L)
{
    VecDesc d = velocity_desc(L);
    d.seg[0].ncomp = 1;
    d.total        = d.seg[0].stride;
    return d;
}

VecDesc stokes_desc(const DeviceLevel& Lu, const DeviceLevel& Lp)
{
    VecDesc d = velocity_desc(Lu);
    d.nseg    = 2;
    d.seg[1].offset = d.total;
    d.seg[1].n      = Lp.nodes();
    d.seg[1].stride = pad64(Lp.nodes());
    d.seg[1].ncomp  = 1;
    d.seg[1].nr     = Lp.nr();
    d.seg[1].owned  = Lp.owned_lat.as<uint8_t>();
    d.seg[1].rdiv   = reciprocal_nr(Lp.nr());
    d.total += d.seg[1].stride;
    return d;
}

template <typename T>
void DVec<T>::alloc(const VecDesc& desc)
{
    d = desc;
    buf.alloc(static_cast<size_t>(desc.total) * sizeof(T));
    cuda_check(cudaMemset(buf.get(), 0, static_cast<size_t>(desc.total) * sizeof(T)), "zero vector");
}
template <typename T>
int DVec<T>::ncomp() const
{
    int n = 0;
    for (int s = 0; s < d.nseg; ++s) n += d.seg[s].ncomp;
    return n;
}
template <typename T>
void DVec<T>::comps(T** out) const
{
    int k = 0;
    for (int s = 0; s < d.nseg; ++s)
        for (int c = 0; c < d.seg[s].ncomp; ++c) out[k++] = comp(s, c);
}
template struct DVec<double>;
template struct DVec<float>;

Scratch::Scratch()
{
    partials.alloc(sizeof(double) * solver_partials_size());
    counter.alloc(sizeof(unsigned));
    scal.alloc(sizeof(double) * kScalars);
    flag.alloc(sizeof(int) * 4);
    cuda_check(cudaMemset(counter.get(), 0, sizeof(unsigned)), "zero counter");
    cuda_check(cudaMemset(scal.get(), 0, sizeof(double) * kScalars), "zero scalars");
    cuda_check(cudaMemset(flag.get(), 0, sizeof(int) * 4), "zero flag");
    cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&host), sizeof(double) * (kScalars + 1), cudaHostAllocDefault),
               "pinned scalars");
    std::memset(host, 0, sizeof(double) * (kScalars + 1));
}

Scratch::~Scratch()
{
    if (host) cudaFreeHost(host);
}

void Scratch::fetch(int n, cudaStream_t st)
{
    if (n > 0)
        cuda_check(cudaMemcpyAsync(host, scal.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st), "fetch scalars");
    cuda_check(cudaMemcpyAsync(host + kScalars, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st), "fetch flag");
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

// ---------------------------------------------------------------------------
// Velocity multigrid
// ---------------------------------------------------------------------------
template <>
VelocityMultigrid::Work<double>& VelocityMultigrid::work<double>()
{
    return w64_;
}
template <>
VelocityMultigrid::Work<float>& VelocityMultigrid::work<float>()
{
    return w32_;
}

VelocityMultigrid::VelocityMultigrid(const Shell* sh, const EpsDivDivOp& fine, const MgOptions& o, Scratch& scratch,
                                     cudaStream_t st)
    : sh_(sh), fine_(fine.level), opt_(o), scratch_(scratch)
{
    if (fine.stored) throw Error(kErrUnsupported, "the finest multigrid operator must be matrix-free");
    if (fine.precision != 0) throw Error(kErrArg, "the multigrid hierarchy is built from an FP64 operator");
    if (fine_ < 1) throw Error(kErrArg, "multigrid needs at least two levels");
    if (o.cheb_order < 1 || o.cheb_iters < 0 || o.num_vcycles < 1 || o.coarse_max_iter < 0 ||
        (o.smoother != 0 && o.smoother != 1) || !(o.jacobi_omega > 0.0) || (o.transfer != 0 && o.transfer != 1))
        throw Error(kErrArg, "invalid multigrid options");
    const int nlev = fine_ + 1;
    ops64_.resize(nlev);
    ops32_.resize(nlev);
    lambda_.assign(nlev, 0.0);

    auto make_op = [&](int l) {
        auto op        = std::make_unique<EpsDivDivOp>();
        op->shell      = sh;
        op->level      = l;
        op->precision  = 0;
        op->apply_mode = 0;
        op->comm_mode  = 1;
        op->bc_cmb     = fine.bc_cmb;
        op->bc_surf    = fine.bc_surf;
        op->q0         = fine.q0;
        return op;
    };
    // finest: copy of the caller's operator
    {
        auto op = make_op(fine_);
        op->k.alloc(fine.k.size());
        cuda_check(cudaMemcpyAsync(op->k.get(), fine.k.get(), fine.k.size(), cudaMemcpyDeviceToDevice, st),
                   "copy coefficient");
        op->tile_y  = fine.tile_y;
        op->chunk_x = fine.chunk_x;
        ops64_[fine_] = std::move(op);
    }
    // adaptive GCA (gca = 2): GCAElementsCollector on the fine coefficient marks coarsest cells
    // (stokes_solver.hpp:278-287)
    DevBuf marks;
    if (o.gca == 2) {
        if (fine.q0) throw Error(kErrUnsupported, "adaptive GCA marks cells from a nodal coefficient");
        const DeviceLevel& L0 = sh->level(0);
        marks.alloc(static_cast<size_t>(L0.cells()));
        cuda_check(cudaMemsetAsync(marks.get(), 0, marks.size(), st), "clear marks");
        const DeviceLevel& Lf = sh->level(fine_);
        chk(gca_mark_elements(Lf.nl(), Lf.nr(), ops64_[fine_]->k.as<double>(), fine_, marks.as<uint8_t>(), st),
            "mark GCA elements");
    }
    // coarse levels: Galerkin (TwoGridGCA top-down, stokes_solver.hpp:375-389) on every cell (gca = 1), on the
    // marked cells only with the rediscretised operator elsewhere (gca = 2, OperatorStoredMatrixMode::Selective,
    // :360-366), or rediscretised (gca = 0)
    for (int l = fine_ - 1; l >= 0; --l) {
        auto op = make_op(l);
        if (o.gca == 1) {
            gca_coarsen(*ops64_[l + 1], *op, st, o.transfer == 1);
        } else {
            const DeviceLevel& Lc = sh->level(l);
            const auto&        kf = ops64_[l + 1]->k;
            if (op->q0) {
                op->k.alloc(sizeof(double) * Lc.cells());
                chk(cell_coefficient_average(Lc.nl(), Lc.nr(), kf.as<double>(), op->k.as<double>(), st), "coarsen");
            } else {
                op->k.alloc(sizeof(double) * Lc.nodes());
                chk(coefficient_inject(Lc.nl(), Lc.nr(), kf.as<double>(), op->k.as<double>(), false, st), "inject");
            }
            if (o.gca == 2) {
                op->set_selective(marks.as<uint8_t>(), l, st);
                gca_coarsen(*ops64_[l + 1], *op, st, o.transfer == 1);
            }
        }
        ops64_[l] = std::move(op);
    }
    // the coarsest CG runs over stored matrices
    ops64_[0]->materialize_full(st);
    if (!ops64_[0]->stored) ops64_[0]->set_stored_matrices_from_coefficient(st);
    ops64_[0]->ensure_baked(false, st);
    {
        const DeviceLevel& L0   = sh->level(0);
        const int          nmem = static_cast<int>(L0.host.dup_members.size());
        chk(coarse_pcg_prepare(L0.nl(), L0.nr(), L0.iface.num_classes, nmem), "coarse CG configuration");
        if (coarse_pcg_uses_full_matrices(L0.nl(), L0.nr(), L0.iface.num_classes, nmem)) {
            const int nc0 = static_cast<int>(L0.cells());
            cfull_.alloc(sizeof(double) * 2 * 324 * static_cast<size_t>(nc0));
            chk(coarse_matrices_unpack(nc0, ops64_[0]->baked64.as<double>(), cfull_.as<double>(), st), "unpack");
            cuda_check(cudaStreamSynchronize(st), "unpack");
        }
    }

    if (o.coarse_dense) build_dense_coarse(st);
    if (o.transfer == 1)  // linear-transfer weights of every fine level, before any stream capture
        for (int l = 1; l <= fine_; ++l) {
            sh->level(l).linear_weights<double>(st);
            if (o.fp32) sh->level(l).linear_weights<float>(st);
        }

    // FP32 operators where the apply is matrix-free
    if (o.fp32) {
        for (int l = 1; l <= fine_; ++l) {
            if (ops64_[l]->stored || ops64_[l]->selective) {
                ops64_[l]->prepare_fp32(st);
                if (ops64_[l]->stored || ops64_[l]->sel_count > 0) ops64_[l]->ensure_baked(true, st);
                continue;
            }
            auto op       = make_op(l);
            op->precision = 1;
            op->tile_y    = ops64_[l]->tile_y;
            op->chunk_x   = ops64_[l]->chunk_x;
            const int64_t n = static_cast<int64_t>(ops64_[l]->k.size() / sizeof(double));
            op->k.alloc(sizeof(float) * n);
            chk(convert_f64_to_f32(n, ops64_[l]->k.as<double>(), op->k.as<float>(), st), "convert coefficient");
            ops32_[l] = std::move(op);
        }
    }

    // work vectors
    auto alloc_work = [&](auto& W, bool all_levels) {
        W.r.resize(nlev);
        W.e.resize(nlev);
        W.tmp.resize(nlev);
        W.d.resize(nlev);
        W.invdiag.resize(nlev);
        for (int l = 0; l < nlev; ++l) {
            const VecDesc vd = velocity_desc(sh->level(l));
            W.r[l].alloc(vd);
            W.e[l].alloc(vd);
            if (l >= 1 || all_levels) {
                W.tmp[l].alloc(vd);
                W.d[l].alloc(vd);
                W.invdiag[l].alloc(vd);
            }
        }
    };
    alloc_work(w64_, false);
    if (o.fp32) alloc_work(w32_, false);

    // inverse diagonals (stokes_solver.hpp:391-417): diagonal mode applied to ones
    for (int l = 1; l <= fine_; ++l) {
        const DeviceLevel& L    = sh->level(l);
        DVec<double>&      ones = w64_.tmp[l];
        DVec<double>&      dg   = w64_.invdiag[l];
        double*            oc[3];
        double*            dc[3];
        ones.comps(oc);
        dg.comps(dc);
        double* o3[3] = {oc[0], oc[1], oc[2]};
        chk(lincomb<double>(L.nodes(), 3, o3, 1.0, 0, nullptr, nullptr, nullptr, nullptr, st), "assign");
        EpsDivDivOp& A = *ops64_[l];
        A.diagonal     = true;
        const double* oc_c[3] = {oc[0], oc[1], oc[2]};
        A.apply_t<double>(oc_c, dc, st);
        A.diagonal = false;
        chk(invert_inplace<double>(L.nodes(), 3, dc, st), "invert");
        if (o.fp32) chk(convert_f64_to_f32(dg.total(), dg.data(), w32_.invdiag[l].data(), st), "convert diagonal");
        chk(lincomb<double>(L.nodes(), 3, o3, 0.0, 0, nullptr, nullptr, nullptr, nullptr, st), "zero");
    }
    // Chebyshev spectrum estimates (chebyshev.hpp estimate_max_eigenvalues)
    // lambda_max of D^-1 A per level for the Chebyshev smoother (the Jacobi smoother needs none)
    if (o.smoother == 0)
        for (int l = 1; l <= fine_; ++l) lambda_[l] = power_iteration(l, o.power_iters, o.seed + 7919ull * l, st);
    // one FP32 apply per level now: kernel attributes are set outside any later graph capture
    if (o.fp32)
        for (int l = 1; l <= fine_; ++l) apply<float>(l, w32_.e[l].data(), w32_.tmp[l].data(), st);

    // coarsest CG vectors
    const VecDesc v0 = velocity_desc(sh->level(0));
    cx_.alloc(v0);
    cb_.alloc(v0);
    cr_.alloc(v0);
    cp_.alloc(v0);
    cap_.alloc(v0);
    cpart_.alloc(sizeof(double) * coarse_pcg_partials_size());
    cstats_.alloc(sizeof(double) * 4);
    cuda_check(cudaMemset(cstats_.get(), 0, sizeof(double) * 4), "zero stats");
}

// Dense inverse of the coarsest operator (coarse_dense.cu): unique-node numbering from the ownership flags and
// the duplicate classes, one column per unknown from the stored operator applied to a unit vector that is 1 on
// every copy of the unknown, then in-place Gauss-Jordan inversion. Synchronous set-up.
void VelocityMultigrid::build_dense_coarse(cudaStream_t st)
{
    const DeviceLevel& L0 = sh_->level(0);
    const ShellLevel&  h  = L0.host;
    const int          nr = L0.nr();
    const int64_t      nodes = L0.nodes();
    const int          nlat  = static_cast<int>(h.owned_lat.size());
    std::vector<int32_t> owner(nlat);
    for (int c = 0; c < nlat; ++c) owner[c] = c;
    for (size_t k = 0; k + 1 < h.dup_offset.size(); ++k) {
        int32_t own = -1;
        for (int32_t m = h.dup_offset[k]; m < h.dup_offset[k + 1]; ++m)
            if (h.owned_lat[h.dup_members[m]]) own = h.dup_members[m];
        if (own < 0) throw Error(kErrState, "a duplicate class without an owned copy");
        for (int32_t m = h.dup_offset[k]; m < h.dup_offset[k + 1]; ++m) owner[h.dup_members[m]] = own;
    }
    std::vector<int32_t> uid_owned(static_cast<size_t>(nodes), -1), rep, uid(static_cast<size_t>(nodes));
    for (int c = 0; c < nlat; ++c)
        if (h.owned_lat[c])
            for (int r = 0; r < nr; ++r) {
                uid_owned[static_cast<size_t>(c) * nr + r] = static_cast<int32_t>(rep.size());
                rep.push_back(static_cast<int32_t>(c * nr + r));
            }
    for (int c = 0; c < nlat; ++c)
        for (int r = 0; r < nr; ++r) uid[static_cast<size_t>(c) * nr + r] = uid_owned[static_cast<size_t>(owner[c]) * nr + r];
    knu_         = static_cast<int>(rep.size());
    const int nd = 3 * knu_;
    if (nd > kDenseCoarseMaxUnknowns)
        throw Error(kErrUnsupported, "the coarsest level is too large for the dense coarse solve (" +
                                         std::to_string(nd) + " unknowns)");
    chk(dense_coarse_prepare(nd), "dense coarse configuration");
    kuid_ = upload(uid);
    krep_ = upload(rep);
    ky_.alloc(sizeof(double) * nd);
    kinv_.alloc(sizeof(double) * static_cast<size_t>(nd) * nd);
    DevBuf        colk(sizeof(double) * nd);
    const VecDesc v0 = velocity_desc(L0);
    DVec<double>  e, y;
    e.alloc(v0);
    y.alloc(v0);
    const int64_t s      = v0.seg[0].stride;
    EpsDivDivOp&  A0     = *ops64_[0];
    const int     amode  = A0.apply_mode, cmode = A0.comm_mode;
    A0.apply_mode        = 0;
    A0.comm_mode         = 1;
    const double* src[3] = {e.data(), e.data() + s, e.data() + 2 * s};
    double*       dst[3] = {y.data(), y.data() + s, y.data() + 2 * s};
    for (int j = 0; j < nd; ++j) {
        chk(dense_unit_vector(nodes, s, knu_, kuid_.as<int32_t>(), j, e.data(), st), "unit vector");
        A0.apply_t<double>(src, dst, st);
        chk(dense_gather_column(knu_, s, krep_.as<int32_t>(), y.data(), j, kinv_.as<double>(), st), "column");
    }
    A0.apply_mode = amode;
    A0.comm_mode  = cmode;
    chk(dense_invert_spd(nd, kinv_.as<double>(), colk.as<double>(), st), "inversion");
    cuda_check(cudaStreamSynchronize(st), "dense coarse set-up");
}

double VelocityMultigrid::power_iteration(int l, int iterations, uint64_t seed, cudaStream_t st)
{
    // it <- seeded start, normalised; aux = D^-1 A it; repeat: it = aux/|aux|, aux = D^-1 A it;
    // radius = <it, aux> (power_iteration.hpp:15-57)
    const DeviceLevel& L   = sh_->level(l);
    DVec<double>&      it  = w64_.e[l];
    DVec<double>&      aux = w64_.d[l];
    const VecDesc      vd  = it.d;
    const int64_t      nt  = vd.total;
    {
        double* ic[3];
        it.comps(ic);
        chk(random_fill<double>(L.nodes(), 3, ic, L.nr(), L.canon_lat.as<int32_t>(), seed, st), "random");
    }
    chk(vec_dot<double>(vd, it.data(), it.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
    chk(scale_by_recip<double>(nt, it.data(), it.data(), scratch_.s(0), st), "scale");
    apply<double>(l, it.data(), aux.data(), st);
    chk(vec_mul<double>(nt, aux.data(), aux.data(), w64_.invdiag[l].data(), 1.0, st), "scale diag");
    for (int k = 0; k < iterations; ++k) {
        chk(vec_dot<double>(vd, aux.data(), aux.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
        chk(scale_by_recip<double>(nt, it.data(), aux.data(), scratch_.s(0), st), "scale");
        apply<double>(l, it.data(), aux.data(), st);
        chk(vec_mul<double>(nt, aux.data(), aux.data(), w64_.invdiag[l].data(), 1.0, st), "scale diag");
    }
    double radius = 0.0;
    if (iterations > 0) {
        chk(vec_dot<double>(vd, it.data(), aux.data(), scratch_.s(1), scratch_.rs(), false, st), "dot");
        scratch_.fetch(2, st);
        radius = scratch_.host[1];
    }
    cuda_check(cudaMemsetAsync(it.data(), 0, sizeof(double) * nt, st), "zero");
    cuda_check(cudaMemsetAsync(aux.data(), 0, sizeof(double) * nt, st), "zero");
    return radius;
}

template <typename T>
void VelocityMultigrid::apply(int l, const T* x, T* y, cudaStream_t st)
{
    const DeviceLevel& L = sh_->level(l);
    const int64_t      s = pad64(L.nodes());
    const T*           src[3] = {x, x + s, x + 2 * s};
    T*                 dst[3] = {y, y + s, y + 2 * s};
    if (std::is_same<T, float>::value && ops32_[l])
        ops32_[l]->apply_t<T>(src, dst, st);
    else
        ops64_[l]->apply_t<T>(src, dst, st);
}

// Chebyshev::solve_impl (chebyshev.hpp:102-176); rho carries over between the
// outer iterations as in the reference. With x_zero (x holds zeros on entry,
// as in every pre-smoothing of a V-cycle that starts from zero) the first
// step's A x is exactly zero and is written as zeros instead of applied.
template <typename T>
void VelocityMultigrid::smooth(int l, T* x, const T* b, cudaStream_t st, bool x_zero)
{
    Work<T>& W = work<T>();
    auto     residual_apply = [&](T* ax, bool first) {
        if (first && x_zero)
            cuda_check(cudaMemsetAsync(ax, 0, sizeof(T) * W.tmp[l].total(), st), "zero");
        else
            apply<T>(l, x, ax, st);
    };
    if (opt_.smoother == 1) {
        // Jacobi::solve_impl (jacobi.hpp:51-60): x += omega D^-1 (b - A x), one
        // fused update per step (the first-step form of the Chebyshev kernel)
        const int64_t n    = W.tmp[l].total();
        T*            ax   = W.tmp[l].data();
        T*            d    = W.d[l].data();
        const T*      invd = W.invdiag[l].data();
        for (int it = 0; it < opt_.cheb_iters; ++it) {
            residual_apply(ax, it == 0);
            chk(cheb_step<T>(n, x, d, b, ax, invd, static_cast<T>(opt_.jacobi_omega), T(0), true, st), "jacobi");
        }
        return;
    }
    double ev = lambda_[l];
    if (!std::isfinite(ev) || ev <= 0.0) ev = 1.0;
    const double  lmax = 1.5 * ev, lmin = 0.1 * ev;
    const double  theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double  sigma = theta / delta;
    double        rho   = 1.0 / sigma;
    const int64_t n     = W.tmp[l].total();
    T*            ax    = W.tmp[l].data();
    T*            d     = W.d[l].data();
    const T*      invd  = W.invdiag[l].data();
    for (int it = 0; it < opt_.cheb_iters; ++it) {
        residual_apply(ax, it == 0);
        chk(cheb_step<T>(n, x, d, b, ax, invd, static_cast<T>(1.0 / theta), T(0), true, st), "chebyshev");
        for (int i = 2; i <= opt_.cheb_order; ++i) {
            const double rho_new = 1.0 / (2.0 * sigma - rho);
            const double beta    = rho_new * rho;
            const double alpha   = 2.0 * rho_new / delta;
            apply<T>(l, x, ax, st);
            chk(cheb_step<T>(n, x, d, b, ax, invd, static_cast<T>(alpha), static_cast<T>(beta), false, st),
                "chebyshev");
            rho = rho_new;
        }
    }
}

// solve_recursive (multigrid.hpp:288-432, classical V-cycle branch)
template <typename T>
void VelocityMultigrid::vcycle(int l, T* x, const T* b, cudaStream_t st, bool x_zero)
{
    if (l == 0) {
        coarse_solve<T>(x, b, st);
        return;
    }
    Work<T>&           W  = work<T>();
    const DeviceLevel& L  = sh_->level(l);
    const DeviceLevel& Lc = sh_->level(l - 1);
    smooth<T>(l, x, b, st, x_zero);
    T* res = W.tmp[l].data();
    apply<T>(l, x, res, st);
    const T one_m[2] = {T(1), T(-1)};
    lin<T>(W.tmp[l].total(), res, T(0), 2, one_m, b, res, st);
    const int64_t sf = pad64(L.nodes()), sc = pad64(Lc.nodes());
    T*            rc = W.r[l - 1].data();
    T*            ec = W.e[l - 1].data();
    const T*      fin[3]  = {res, res + sf, res + 2 * sf};
    T*            cout[3] = {rc, rc + sc, rc + 2 * sc};
    if (opt_.transfer == 1)
        chk(restrict_linear_owned<T>(L.nl(), L.nr(), 3, L.owned_lat.as<uint8_t>(), L.linear_weights<T>(st), fin,
                                     cout, st),
            "restrict");
    else
        chk(restrict_owned<T>(L.nl(), L.nr(), 3, L.owned_lat.as<uint8_t>(), fin, cout, st), "restrict");
    chk(interface_sum<T>(Lc.iface, Lc.nr(), 3, cout, st), "interface sum");
    cuda_check(cudaMemsetAsync(ec, 0, sizeof(T) * W.e[l - 1].total(), st), "zero correction");
    vcycle<T>(l - 1, ec, rc, st, true);
    const T* cin[3]  = {ec, ec + sc, ec + 2 * sc};
    T*       fout[3] = {x, x + sf, x + 2 * sf};
    if (opt_.transfer == 1)
        chk(prolongate_linear_add<T>(L.nl(), L.nr(), 3, L.linear_weights<T>(st), cin, fout, st), "prolongate");
    else
        chk(prolongate_add<T>(L.nl(), L.nr(), 3, cin, fout, st), "prolongate");
    smooth<T>(l, x, b, st, false);
}

template <typename T>
void VelocityMultigrid::coarse_solve(T* x, const T* b, cudaStream_t st)
{
    const DeviceLevel& L0 = sh_->level(0);
    const int64_t      nt = cx_.total();
    double*            xd;
    const double*      bd;
    if (std::is_same<T, double>::value) {
        xd = reinterpret_cast<double*>(x);
        bd = reinterpret_cast<const double*>(b);
    } else {
        chk(convert_f32_to_f64(nt, reinterpret_cast<const float*>(x), cx_.data(), st), "widen");
        chk(convert_f32_to_f64(nt, reinterpret_cast<const float*>(b), cb_.data(), st), "widen");
        xd = cx_.data();
        bd = cb_.data();
    }
    if (kinv_.get() != nullptr) {
        chk(dense_coarse_solve(L0.nodes(), pad64(L0.nodes()), knu_, kuid_.as<int32_t>(), krep_.as<int32_t>(),
                               kinv_.as<double>(), bd, ky_.as<double>(), xd, st),
            "dense coarse solve");
        if (!std::is_same<T, double>::value)
            chk(convert_f64_to_f32(nt, cx_.data(), reinterpret_cast<float*>(x), st), "narrow");
        return;
    }
    EpsDivDivOp& A0 = *ops64_[0];
    A0.ensure_baked(false, st);
    CoarsePcgArgs a;
    a.nl          = L0.nl();
    a.nr          = L0.nr();
    a.mats        = A0.baked64.as<double>();
    a.mats_full   = cfull_.size() ? cfull_.as<double>() : nullptr;
    a.num_classes = L0.iface.num_classes;
    a.num_members = static_cast<int>(L0.host.dup_members.size());
    a.off         = L0.iface.offset;
    a.mem         = L0.iface.members;
    a.owned       = L0.owned_lat.as<uint8_t>();
    a.n           = L0.nodes();
    a.stride      = pad64(L0.nodes());
    a.x           = xd;
    a.b           = bd;
    a.r           = cr_.data();
    a.p           = cp_.data();
    a.ap          = cap_.data();
    a.partials    = cpart_.as<double>();
    a.max_iter    = opt_.coarse_max_iter;
    a.rtol        = opt_.coarse_rtol;
    a.atol        = opt_.coarse_atol;
    a.stats       = cstats_.as<double>();
    chk(coarse_pcg(a, st), "coarse CG");
    if (!std::is_same<T, double>::value)
        chk(convert_f64_to_f32(nt, cx_.data(), reinterpret_cast<float*>(x), st), "narrow");
}

void VelocityMultigrid::solve64(double* x, const double* b, cudaStream_t st, bool x_zero)
{
    for (int c = 0; c < opt_.num_vcycles; ++c) vcycle<double>(fine_, x, b, st, x_zero && c == 0);
}

void VelocityMultigrid::solve32(float* x, const float* b, cudaStream_t st, bool x_zero)
{
    if (!opt_.fp32) throw Error(kErrState, "the hierarchy was built without FP32 operators");
    for (int c = 0; c < opt_.num_vcycles; ++c) vcycle<float>(fine_, x, b, st, x_zero && c == 0);
}

template <typename T>
void VelocityMultigrid::solve_external(T* const* x, const T* const* b, cudaStream_t st)
{
    const DeviceLevel& L  = sh_->level(fine_);
    const VecDesc      vd = velocity_desc(L);
    auto&              ex = [this]() -> auto& {
        if constexpr (std::is_same<T, double>::value)
            return ext64_;
        else
            return ext32_;
    }();
    if (ex[0].buf.get() == nullptr) {
        ex[0].alloc(vd);
        ex[1].alloc(vd);
    }
    const size_t bytes = sizeof(T) * L.nodes();
    for (int c = 0; c < 3; ++c) {
        cuda_check(cudaMemcpyAsync(ex[0].comp(0, c), x[c], bytes, cudaMemcpyDeviceToDevice, st), "copy in");
        cuda_check(cudaMemcpyAsync(ex[1].comp(0, c), b[c], bytes, cudaMemcpyDeviceToDevice, st), "copy in");
    }
    if constexpr (std::is_same<T, double>::value)
        solve64(ex[0].data(), ex[1].data(), st);
    else
        solve32(ex[0].data(), ex[1].data(), st);
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(x[c], ex[0].comp(0, c), bytes, cudaMemcpyDeviceToDevice, st), "copy out");
}
template void VelocityMultigrid::solve_external<double>(double* const*, const double* const*, cudaStream_t);
template void VelocityMultigrid::solve_external<float>(float* const*, const float* const*, cudaStream_t);

void VelocityMultigrid::coarse_stats(double* out3, cudaStream_t st)
{
    cuda_check(cudaMemcpyAsync(out3, cstats_.get(), sizeof(double) * 3, cudaMemcpyDeviceToHost, st), "stats");
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

// ---------------------------------------------------------------------------
// Stokes FGMRES
// ---------------------------------------------------------------------------
StokesSolver::StokesSolver(const Shell* sh, int vlevel, const double* eta_nodal, const double* eta_cell,
                           const double* k_schur, int bc_cmb, int bc_surf, const StokesOptions& o, cudaStream_t st)
    : sh_(sh), vlevel_(vlevel), opt_(o)
{
    if ((eta_nodal == nullptr) == (eta_cell == nullptr))
        throw Error(kErrArg, "exactly one of eta_nodal / eta_cell must be given");
    if (vlevel < 1) throw Error(kErrArg, "the velocity level needs a pressure level below it");
    if (o.restart < 1 || o.restart > kMaxAxpy || o.restart + 2 > Scratch::kScalars || o.max_iter < 0)
        throw Error(kErrArg, "FGMRES restart must be in 1..128");
    if (eta_cell && !k_schur) throw Error(kErrArg, "a cell viscosity needs the Schur coefficient k_schur");
    const DeviceLevel& Lu = sh->level(vlevel);
    const DeviceLevel& Lp = sh->level(vlevel - 1);

    auto setup = [&](Operator& op) {
        op.shell      = sh;
        op.level      = vlevel;
        op.precision  = 0;
        op.apply_mode = 0;
        op.comm_mode  = 1;
        op.bc_cmb     = bc_cmb;
        op.bc_surf    = bc_surf;
    };
    setup(K_);
    setup(K_.A);
    setup(K_.B);
    setup(K_.BT);
    setup(BT_);
    K_.A.q0              = eta_cell != nullptr;
    const size_t kbytes  = sizeof(double) * (K_.A.q0 ? Lu.cells() : Lu.nodes());
    K_.A.k.alloc(kbytes);
    cuda_check(cudaMemcpyAsync(K_.A.k.get(), K_.A.q0 ? static_cast<const void*>(eta_cell) : eta_nodal, kbytes,
                               cudaMemcpyDeviceToDevice, st),
               "copy viscosity");

    // Schur block: lumped KMass with k = 1/eta on the pressure level, inverted (DiagonalSolver)
    inv_schur_.alloc(scalar_desc(Lp));
    {
        DevBuf kp(sizeof(double) * Lp.nodes());
        if (k_schur)
            cuda_check(cudaMemcpyAsync(kp.get(), k_schur, sizeof(double) * Lp.nodes(), cudaMemcpyDeviceToDevice, st),
                       "copy k_schur");
        else
            chk(coefficient_inject(Lp.nl(), Lp.nr(), eta_nodal, kp.as<double>(), true, st), "schur coefficient");
        double* dg = inv_schur_.data();
        chk(kmass_lumped_add<double>(Lp.nl(), Lp.nr(), Lp.coords<double>(), Lp.radii<double>(), kp.as<double>(), dg, st),
            "kmass");
        chk(interface_sum<double>(Lp.iface, Lp.nr(), 1, &dg, st), "interface sum");
        chk(invert_inplace<double>(Lp.nodes(), 1, &dg, st), "invert");
        cuda_check(cudaStreamSynchronize(st), "synchronize");
    }

    MgOptions mo = o.mg;
    mg_          = std::make_unique<VelocityMultigrid>(sh, K_.A, mo, scratch_, st);
    ones_p_.alloc(scalar_desc(Lp));
    {
        double* oc[1] = {ones_p_.data()};
        chk(lincomb<double>(Lp.nodes(), 1, oc, 1.0, 0, nullptr, nullptr, nullptr, nullptr, st), "ones");
        num_owned_p_ = 0;
        for (auto o8 : Lp.host.owned_lat) num_owned_p_ += o8;
        num_owned_p_ *= Lp.nr();
    }

    blk_ = stokes_desc(Lu, Lp);
    x_.alloc(blk_);
    b_.alloc(blk_);
    r_.alloc(blk_);
    w_.alloc(blk_);
    t_.alloc(velocity_desc(Lu));
    V_.resize(o.restart + 1);
    Z_.resize(o.restart);
    for (auto& v : V_) v.alloc(blk_);
    for (auto& z : Z_) z.alloc(blk_);
    if (mo.fp32) {
        t32_.alloc(velocity_desc(Lu));
        z32_.alloc(velocity_desc(Lu));
    }
    // everything an Arnoldi step touches is allocated here, so that the step can be captured
    const size_t wedges = sizeof(double) * 2 * static_cast<size_t>(Lu.cells());
    K_.B.scratch.alloc(wedges);
    K_.BT.scratch.alloc(wedges);
    BT_.scratch.alloc(wedges);
    graphs_.assign(o.restart, nullptr);
    graph_kernels_.assign(o.restart, 0);
    cuda_check(cudaStreamCreateWithFlags(&ws_, cudaStreamNonBlocking), "create stream");
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

void StokesSolver::stokes_apply(const DVec<double>& x, DVec<double>& y, cudaStream_t st)
{
    double* xs[4];
    double* ys[4];
    x.comps(xs);
    y.comps(ys);
    void* const src[4] = {xs[0], xs[1], xs[2], xs[3]};
    void* const dst[4] = {ys[0], ys[1], ys[2], ys[3]};
    K_.apply(src, dst, st);
}

// BlockTriangularPreconditioner2x2::solve_impl: z_p = S^-1 v_p; t = B^T z_p + v_u;
// z_p = -z_p; z_u = MG(t) from z_u = 0. Sets the scratch flag when z has a
// NaN or Inf.
void StokesSolver::precondition(const DVec<double>& v, DVec<double>& z, cudaStream_t st)
{
    const VecSeg& su = blk_.seg[0];
    const VecSeg& sp = blk_.seg[1];
    double*       zp = z.data() + sp.offset;
    chk(vec_mul<double>(sp.stride, zp, v.data() + sp.offset, inv_schur_.data(), 1.0, st), "schur");
    {
        void* const src[1] = {zp};
        double*     tc[3];
        t_.comps(tc);
        void* const dst[3] = {tc[0], tc[1], tc[2]};
        BT_.apply_mode     = 0;
        BT_.comm_mode      = 1;
        BT_.apply(src, dst, st);
    }
    const double one_one[2] = {1.0, 1.0};
    lin<double>(t_.total(), t_.data(), 0.0, 2, one_one, t_.data(), v.data() + su.offset, st);
    const double neg[1] = {-1.0};
    lin<double>(sp.stride, zp, 0.0, 1, neg, zp, nullptr, st);
    if (opt_.mg.fp32) {
        chk(convert_f64_to_f32(t_.total(), t_.data(), t32_.data(), st), "narrow");
        cuda_check(cudaMemsetAsync(z32_.data(), 0, sizeof(float) * z32_.total(), st), "zero");
        mg_->solve32(z32_.data(), t32_.data(), st, true);
        chk(widen_check(z32_.total(), z32_.data(), z.data() + su.offset, scratch_.flag_dev(), st), "widen");
        chk(flag_nonfinite<double>(sp.stride, zp, scratch_.flag_dev(), st), "check");
    } else {
        mg_->solve64(z.data() + su.offset, t_.data(), st, true);  // both callers pass z = 0
        chk(flag_nonfinite<double>(z.total(), z.data(), scratch_.flag_dev(), st), "check");
    }
}

void StokesSolver::copy_in(DVec<double>& v, const double* const* u, const double* p, cudaStream_t st)
{
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(v.comp(0, c), u[c], sizeof(double) * blk_.seg[0].n, cudaMemcpyDeviceToDevice, st),
                   "copy in");
    cuda_check(cudaMemcpyAsync(v.comp(1, 0), p, sizeof(double) * blk_.seg[1].n, cudaMemcpyDeviceToDevice, st),
               "copy in");
}

void StokesSolver::copy_out(const DVec<double>& v, double* const* u, double* p, cudaStream_t st)
{
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(u[c], v.comp(0, c), sizeof(double) * blk_.seg[0].n, cudaMemcpyDeviceToDevice, st),
                   "copy out");
    cuda_check(cudaMemcpyAsync(p, v.comp(1, 0), sizeof(double) * blk_.seg[1].n, cudaMemcpyDeviceToDevice, st),
               "copy out");
}

// v_p -= (sum of v_p over owned pressure nodes) / (number of owned pressure nodes)
void StokesSolver::remove_pressure_mean(DVec<double>& v, int slot, cudaStream_t st)
{
    const VecSeg& sp = blk_.seg[1];
    const VecDesc pd = scalar_desc(sh_->level(vlevel_ - 1));
    chk(vec_dot<double>(pd, v.data() + sp.offset, ones_p_.data(), scratch_.s(slot), scratch_.rs(), false, st), "sum");
    chk(sub_scalar(sp.n, v.data() + sp.offset, scratch_.s(slot), 1.0 / static_cast<double>(num_owned_p_), st),
        "shift");
}

void StokesSolver::precondition_external(const double* const* v, double* const* z, cudaStream_t st)
{
    copy_in(r_, v, v[3], st);
    cuda_check(cudaMemsetAsync(w_.data(), 0, sizeof(double) * w_.total(), st), "zero");
    precondition(r_, w_, st);
    copy_out(w_, z, z[3], st);
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

bool StokesSolver::solve(double* const* u, double* p, const double* const* fu, const double* fp, cudaStream_t st)
{
    // the caller's producers first, then everything on the solver's own stream
    // (graph capture needs a stream other than the legacy default stream)
    cuda_check(cudaStreamSynchronize(st), "synchronize");
    copy_in(x_, u, p, ws_);
    copy_in(b_, fu, fp, ws_);
    const bool ok = solve_internal(ws_);
    copy_out(x_, u, p, ws_);
    cuda_check(cudaStreamSynchronize(ws_), "synchronize");
    return ok;
}

bool StokesSolver::misfit_gradient(const double* const* x, const double* const* u_obs, double* grad_cell,
                                   double* const* lambda, cudaStream_t caller)
{
    cuda_check(cudaStreamSynchronize(caller), "synchronize");
    cudaStream_t st = ws_;
    if (!K_.A.q0) throw Error(kErrUnsupported, "the log-viscosity gradient needs a per-cell viscosity");
    const DeviceLevel& Lu = sh_->level(vlevel_);
    const size_t       bu = sizeof(double) * Lu.nodes();
    // adjoint right-hand side [u - u_obs; 0], boundary rows enforced
    cuda_check(cudaMemsetAsync(b_.data(), 0, sizeof(double) * b_.total(), st), "zero");
    for (int c = 0; c < 3; ++c) {
        double*       y[1]  = {b_.comp(0, c)};
        const double* x0[1] = {x[c]};
        const double* x1[1] = {u_obs[c]};
        const double  cf[2] = {1.0, -1.0};
        chk(lincomb<double>(Lu.nodes(), 1, y, 0.0, 2, cf, x0, x1, nullptr, st), "misfit");
    }
    {
        double* bc[3] = {b_.comp(0, 0), b_.comp(0, 1), b_.comp(0, 2)};
        chk(enforce_velocity_bcs(Lu.nl(), Lu.nr(), Lu.coords<double>(), K_.A.bc_cmb, K_.A.bc_surf, bc, st), "bcs");
    }
    cuda_check(cudaMemsetAsync(x_.data(), 0, sizeof(double) * x_.total(), st), "zero");
    const bool ok = solve_internal(st);
    // grad = -lambda_u^T dA/dlog(eta) u
    const double* uu[3] = {x[0], x[1], x[2]};
    const double* ll[3] = {x_.comp(0, 0), x_.comp(0, 1), x_.comp(0, 2)};
    K_.A.vjp_logeta<double>(uu, ll, grad_cell, st);
    {
        double*       g[1]  = {grad_cell};
        const double* gi[1] = {grad_cell};
        const double  neg   = -1.0;
        chk(lincomb<double>(Lu.cells(), 1, g, 0.0, 1, &neg, gi, nullptr, nullptr, st), "negate");
    }
    if (lambda) {
        for (int c = 0; c < 3; ++c)
            cuda_check(cudaMemcpyAsync(lambda[c], x_.comp(0, c), bu, cudaMemcpyDeviceToDevice, st), "copy out");
        cuda_check(cudaMemcpyAsync(lambda[3], x_.comp(1, 0), sizeof(double) * blk_.seg[1].n, cudaMemcpyDeviceToDevice,
                                   st),
                   "copy out");
    }
    cuda_check(cudaStreamSynchronize(st), "synchronize");
    return ok;
}

// Device work of Arnoldi step j without any host synchronisation:
// V_j = w / h_{j,j-1} (j > 0), Z_j = M^-1 V_j, w = K Z_j, Gram-Schmidt of w
// against V_0..V_j and its norm into the scalar slots. With CUDA graphs on,
// each j is captured once (its pointers are fixed) and replayed.
void StokesSolver::step_body(int j, cudaStream_t st)
{
    const int64_t nt = blk_.total;
    if (j > 0) chk(scale_by_recip<double>(nt, V_[j].data(), w_.data(), scratch_.s(kH0 + j), st), "scale");
    DVec<double>& Zj = Z_[j];
    cuda_check(cudaMemsetAsync(Zj.data(), 0, sizeof(double) * nt, st), "zero");
    precondition(V_[j], Zj, st);
    if (opt_.project_pressure_mean) remove_pressure_mean(Zj, kProj, st);
    arnoldi_tail(j, st);
}

void StokesSolver::arnoldi_tail(int j, cudaStream_t st)
{
    stokes_apply(Z_[j], w_, st);
    if (opt_.project_pressure_mean) remove_pressure_mean(w_, kProj, st);
    for (int i = 0; i <= j; ++i)
        chk(mgs_step(blk_, w_.data(), i > 0 ? V_[i - 1].data() : nullptr, scratch_.s(kH0 + i - 1), V_[i].data(),
                     scratch_.s(kH0 + i), scratch_.rs(), st),
            "gram-schmidt");
    chk(mgs_step(blk_, w_.data(), V_[j].data(), scratch_.s(kH0 + j), nullptr, scratch_.s(kH0 + j + 1), scratch_.rs(),
                 st),
        "gram-schmidt");
}

void StokesSolver::run_step(int j, cudaStream_t st)
{
    if (!opt_.use_graphs) {
        step_body(j, st);
        return;
    }
    if (graphs_[j] == nullptr) {
        cudaGraph_t    g  = nullptr;
        const uint64_t l0 = launch_count();
        cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            step_body(j, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        cuda_check(cudaStreamEndCapture(st, &g), "end capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e  = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "instantiate graph");
        graphs_[j]        = exec;
        graph_kernels_[j] = static_cast<int>(launch_count() - l0);
        note_launch(-graph_kernels_[j]);  // counted again below, when they run
    }
    cuda_check(cudaGraphLaunch(graphs_[j], st), "graph launch");
    note_launch(graph_kernels_[j]);
}

StokesSolver::~StokesSolver()
{
    for (auto& g : graphs_)
        if (g) cudaGraphExecDestroy(g);
    if (ws_) cudaStreamDestroy(ws_);
}

bool StokesSolver::solve_internal(cudaStream_t st)
{
    const double eps   = std::numeric_limits<double>::epsilon();
    const int    m     = opt_.restart;
    const int64_t nt   = blk_.total;
    history.clear();
    iterations   = 0;
    converged    = false;
    final_relres = 0.0;
    cuda_check(cudaMemsetAsync(scratch_.counter.get(), 0, sizeof(unsigned), st), "zero counter");
    cuda_check(cudaMemsetAsync(scratch_.flag_dev(), 0, sizeof(int), st), "zero flag");

    // With project_pressure_mean the iteration runs on P K P with P removing
    // the pressure mean (constant pressure treated as a null vector): with a
    // free-slip surface the divergence rows keep a uniform part
    // 1^T B u = (B^T 1)^T u != 0 (nodal normals are not the facet normals) that
    // the preconditioned system cannot reduce, so the unprojected residual
    // floors at an O(h^2) level. full_relres reports the unprojected residual.
    const double one_m[2] = {1.0, -1.0};
    const int    kFull    = Scratch::kScalars - 2;  // scalar slots away from the Hessenberg column
    static_assert(Scratch::kScalars - 1 == kProj, "projection scratch slot");
    auto residual = [&](bool report_full) {  // r = b - K x, returns ||r|| (projected when enabled)
        stokes_apply(x_, r_, st);
        lin<double>(nt, r_.data(), 0.0, 2, one_m, b_.data(), r_.data(), st);
        if (report_full)
            chk(vec_dot<double>(blk_, r_.data(), r_.data(), scratch_.s(kFull), scratch_.rs(), true, st), "norm");
        if (opt_.project_pressure_mean) remove_pressure_mean(r_, kProj, st);
        chk(vec_dot<double>(blk_, r_.data(), r_.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
        scratch_.fetch(Scratch::kScalars, st);
        return scratch_.host[0];
    };
    // the iterate's pressure stays mean-free under the projection, so the
    // iteration is on [A, B^T P; P B, 0] over mean-free pressures, which is
    // symmetric and nonsingular (the solution is a function of the data)
    if (opt_.project_pressure_mean) remove_pressure_mean(x_, kProj, st);
    double       beta0 = residual(true);
    const double init_full = scratch_.host[kFull];
    const double init  = beta0;
    history.push_back(1.0);
    full_relres = 1.0;
    if (beta0 <= opt_.atol || !(init > 0.0)) {
        converged = true;
        return true;
    }
    std::vector<double> H((m + 1) * m), g(m + 1), cs(m + 1), sn(m + 1), y(m);
    auto                h = [&](int i, int j) -> double& { return H[i * m + j]; };
    int                 total = 0, steps = 0;
    const int           H0    = kH0;  // device scalar slots: s(0) norm scratch, s(H0 + i) Hessenberg column
    while (total < opt_.max_iter) {
        chk(scale_by_recip<double>(nt, V_[0].data(), r_.data(), scratch_.s(0), st), "scale");
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        std::fill(cs.begin(), cs.end(), 0.0);
        std::fill(sn.begin(), sn.end(), 0.0);
        g[0]      = beta0;
        int inner = 0;
        // every Arnoldi step counts toward max_iter when it starts, so a cycle
        // that ends early (the estimate met the tolerance while the recomputed
        // residual did not, a breakdown, stagnation) still makes the loop end
        for (int j = 0; j < m && total < opt_.max_iter; ++j) {
            DVec<double>& Zj = Z_[j];
            ++steps;
            ++total;
            run_step(j, st);
            scratch_.fetch(H0 + j + 2, st);
            if (scratch_.host_flag() != 0) {
                // the preconditioner produced NaN/Inf: keep its input instead (fgmres.hpp:191-210)
                cuda_check(cudaMemsetAsync(scratch_.flag_dev(), 0, sizeof(int), st), "zero flag");
                cuda_check(cudaMemcpyAsync(Zj.data(), V_[j].data(), sizeof(double) * nt, cudaMemcpyDeviceToDevice, st),
                           "copy");
                arnoldi_tail(j, st);
                scratch_.fetch(H0 + j + 2, st);
            }
            for (int i = 0; i <= j; ++i) h(i, j) = scratch_.host[H0 + i];
            const double hj1 = scratch_.host[H0 + j + 1];
            if (hj1 < eps * init) {  // Arnoldi breakdown
                h(j + 1, j) = 0.0;
                inner       = j + 1;
                break;
            }
            h(j + 1, j) = hj1;  // V_{j+1} = w / h_{j+1,j} opens the next step
            for (int i = 0; i < j; ++i) {
                const double t = cs[i] * h(i, j) + sn[i] * h(i + 1, j);
                h(i + 1, j)    = -sn[i] * h(i, j) + cs[i] * h(i + 1, j);
                h(i, j)        = t;
            }
            const double a = h(j, j), bb = h(j + 1, j);
            const double rab = std::hypot(a, bb);
            cs[j]            = rab == 0.0 ? 1.0 : a / rab;
            sn[j]            = rab == 0.0 ? 0.0 : bb / rab;
            h(j, j)          = rab;
            h(j + 1, j)      = 0.0;
            if (std::abs(h(j, j)) < eps) {  // stagnation
                inner = j;
                break;
            }
            const double gj = g[j], gj1 = g[j + 1];
            g[j]               = cs[j] * gj + sn[j] * gj1;
            g[j + 1]           = -sn[j] * gj + cs[j] * gj1;
            const double abs_r = std::abs(g[j + 1]);
            history.push_back(abs_r / init);
            if (!std::isfinite(abs_r)) {
                inner = j;
                break;
            }
            inner = j + 1;
            if (abs_r / init <= opt_.rtol || abs_r < opt_.atol) break;
        }
        for (int row = inner - 1; row >= 0; --row) {
            double s = g[row];
            for (int col = row + 1; col < inner; ++col) s -= h(row, col) * y[col];
            y[row] = s / h(row, row);
        }
        if (inner > 0) {
            AxpyList L;
            L.m = inner;
            for (int i = 0; i < inner; ++i) {
                L.z[i] = Z_[i].data();
                L.y[i] = y[i];
            }
            chk(multi_axpy(nt, x_.data(), L, st), "update");
        }
        beta0        = residual(true);
        final_relres = beta0 / init;
        full_relres  = init_full > 0.0 ? scratch_.host[kFull] / init_full : 0.0;
        if (!std::isfinite(beta0)) break;
        if (beta0 <= opt_.atol || beta0 / init <= opt_.rtol) {
            converged = true;
            break;
        }
    }
    iterations = steps;  // Arnoldi steps (preconditioner applications)
    // "Normalize" pressure: subtract the mean over owned pressure nodes
    // (StokesContext::solve, stokes_solver.hpp:684-690)
    if (opt_.normalize_pressure) {
        const VecSeg& sp = blk_.seg[1];
        VecDesc       pd = scalar_desc(sh_->level(vlevel_ - 1));
        chk(vec_dot<double>(pd, x_.data() + sp.offset, ones_p_.data(), scratch_.s(0), scratch_.rs(), false, st), "sum");
        scratch_.fetch(1, st);
        const double mean  = scratch_.host[0] / static_cast<double>(num_owned_p_);
        double*      pc[1] = {x_.data() + sp.offset};
        const double one   = 1.0;
        const double* src[1] = {x_.data() + sp.offset};
        chk(lincomb<double>(sp.n, 1, pc, -mean, 1, &one, src, nullptr, nullptr, st), "normalise");
    }
    return converged;
}

// ---------------------------------------------------------------------------
// Velocity PCG
// ---------------------------------------------------------------------------
VelocitySolver::VelocitySolver(const Shell* sh, int level, const double* eta_nodal, const double* eta_cell,
                               int bc_cmb, int bc_surf, const VelocitySolverOptions& o, cudaStream_t st)
    : sh_(sh), opt_(o)
{
    if ((eta_nodal == nullptr) == (eta_cell == nullptr))
        throw Error(kErrArg, "exactly one of eta_nodal / eta_cell must be given");
    if (o.max_iter < 0) throw Error(kErrArg, "invalid iteration limit");
    const DeviceLevel& L = sh->level(level);
    A_.shell             = sh;
    A_.level             = level;
    A_.precision         = 0;
    A_.apply_mode        = 0;
    A_.comm_mode         = 1;
    A_.bc_cmb            = bc_cmb;
    A_.bc_surf           = bc_surf;
    A_.q0                = eta_cell != nullptr;
    const size_t kbytes  = sizeof(double) * (A_.q0 ? L.cells() : L.nodes());
    A_.k.alloc(kbytes);
    cuda_check(cudaMemcpyAsync(A_.k.get(), A_.q0 ? static_cast<const void*>(eta_cell) : eta_nodal, kbytes,
                               cudaMemcpyDeviceToDevice, st),
               "copy viscosity");
    mg_ = std::make_unique<VelocityMultigrid>(sh, A_, o.mg, scratch_, st);
    vd_ = velocity_desc(L);
    x_.alloc(vd_);
    b_.alloc(vd_);
    r_.alloc(vd_);
    z_.alloc(vd_);
    p_.alloc(vd_);
    ap_.alloc(vd_);
    if (o.mg.fp32) {
        r32_.alloc(vd_);
        z32_.alloc(vd_);
    }
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

// z = MG(r) from z = 0. The reference's CG hands its previous z to the
// preconditioner as the initial guess (pcg.hpp:150, solve(preconditioner_, A,
// z_, r_)); with a multigrid preconditioner that makes the preconditioner
// non-stationary and CG stalls (the oracle stagnates near 2e-2 at level 3), so
// each application starts from zero here.
void VelocitySolver::precondition(cudaStream_t st)
{
    cuda_check(cudaMemsetAsync(z_.data(), 0, sizeof(double) * z_.total(), st), "zero");
    if (opt_.mg.fp32) {
        chk(convert_f64_to_f32(r_.total(), r_.data(), r32_.data(), st), "narrow");
        cuda_check(cudaMemsetAsync(z32_.data(), 0, sizeof(float) * z32_.total(), st), "zero");
        mg_->solve32(z32_.data(), r32_.data(), st, true);
        chk(convert_f32_to_f64(z_.total(), z32_.data(), z_.data(), st), "widen");
    } else {
        mg_->solve64(z_.data(), r_.data(), st, true);
    }
}

void VelocitySolver::precondition_external(const double* const* v, double* const* z, cudaStream_t st)
{
    const size_t bytes = sizeof(double) * vd_.seg[0].n;
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(r_.comp(0, c), v[c], bytes, cudaMemcpyDeviceToDevice, st), "copy in");
    precondition(st);
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(z[c], z_.comp(0, c), bytes, cudaMemcpyDeviceToDevice, st), "copy out");
    cuda_check(cudaStreamSynchronize(st), "synchronize");
}

bool VelocitySolver::solve(double* const* u, const double* const* f, cudaStream_t st)
{
    const int64_t nt    = vd_.total;
    const size_t  bytes = sizeof(double) * vd_.seg[0].n;
    history.clear();
    iterations   = 0;
    converged    = false;
    final_relres = 0.0;
    cuda_check(cudaMemsetAsync(scratch_.counter.get(), 0, sizeof(unsigned), st), "zero counter");
    for (int c = 0; c < 3; ++c) {
        cuda_check(cudaMemcpyAsync(x_.comp(0, c), u[c], bytes, cudaMemcpyDeviceToDevice, st), "copy in");
        cuda_check(cudaMemcpyAsync(b_.comp(0, c), f[c], bytes, cudaMemcpyDeviceToDevice, st), "copy in");
    }
    auto apply = [&](const DVec<double>& src, DVec<double>& dst) {
        double* sc[3];
        double* dc[3];
        src.comps(sc);
        dst.comps(dc);
        const double* scc[3] = {sc[0], sc[1], sc[2]};
        A_.apply_t<double>(scc, dc, st);
    };
    // r = b - A x; z = M r; p = z
    apply(x_, r_);
    const double one_m[2] = {1.0, -1.0};
    lin<double>(nt, r_.data(), 0.0, 2, one_m, b_.data(), r_.data(), st);
    if (opt_.multigrid_only) {
        // Multigrid::solve_impl with statistics (multigrid.hpp:233-279): residual before and after each cycle
        chk(vec_dot<double>(vd_, r_.data(), r_.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
        scratch_.fetch(1, st);
        const double init = scratch_.host[0];
        history.push_back(1.0);
        converged = init < opt_.atol;
        for (int it = 1; it <= opt_.max_iter && !converged; ++it) {
            mg_->solve64(x_.data(), b_.data(), st);
            apply(x_, r_);
            lin<double>(nt, r_.data(), 0.0, 2, one_m, b_.data(), r_.data(), st);
            chk(vec_dot<double>(vd_, r_.data(), r_.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
            scratch_.fetch(1, st);
            const double res = scratch_.host[0];
            iterations       = it;
            final_relres     = init > 0.0 ? res / init : 0.0;
            history.push_back(final_relres);
            if (!std::isfinite(res)) break;
            converged = final_relres <= opt_.rtol || res < opt_.atol;
        }
        for (int c = 0; c < 3; ++c)
            cuda_check(cudaMemcpyAsync(u[c], x_.comp(0, c), bytes, cudaMemcpyDeviceToDevice, st), "copy out");
        cuda_check(cudaStreamSynchronize(st), "synchronize");
        return converged;
    }
    precondition(st);
    cuda_check(cudaMemcpyAsync(p_.data(), z_.data(), sizeof(double) * nt, cudaMemcpyDeviceToDevice, st), "copy");
    chk(vec_dot<double>(vd_, r_.data(), r_.data(), scratch_.s(0), scratch_.rs(), true, st), "norm");
    scratch_.fetch(1, st);
    const double init = scratch_.host[0];
    history.push_back(1.0);
    // device scalars: s1 = <z, r> (alpha numerator), s2 = <Ap, p>, s3 = |r|, s4 = <z, r> new
    if (init < opt_.atol) {
        converged = true;
    } else {
        chk(vec_dot<double>(vd_, z_.data(), r_.data(), scratch_.s(1), scratch_.rs(), false, st), "dot");
        for (int it = 1; it <= opt_.max_iter; ++it) {
            apply(p_, ap_);
            chk(vec_dot<double>(vd_, ap_.data(), p_.data(), scratch_.s(2), scratch_.rs(), false, st), "dot");
            chk(cg_update(vd_, x_.data(), r_.data(), p_.data(), ap_.data(), scratch_.s(1), scratch_.s(2),
                          scratch_.s(3), scratch_.rs(), st),
                "update");
            scratch_.fetch(4, st);
            const double an = scratch_.host[1], res = scratch_.host[3];
            iterations      = it;
            if (res < 0.0) break;  // |<Ap, p>| below DBL_MIN: no update was made
            const double rel = res / init;
            history.push_back(rel);
            final_relres = rel;
            if (rel <= opt_.rtol || res < opt_.atol) {
                converged = true;
                break;
            }
            precondition(st);
            chk(vec_dot<double>(vd_, z_.data(), r_.data(), scratch_.s(4), scratch_.rs(), false, st), "dot");
            if (std::abs(an) < std::numeric_limits<double>::min()) break;
            chk(p_update(nt, p_.data(), z_.data(), scratch_.s(4), scratch_.s(1), st), "update");
            cuda_check(cudaMemcpyAsync(scratch_.s(1), scratch_.s(4), sizeof(double), cudaMemcpyDeviceToDevice, st),
                       "copy scalar");
        }
    }
    for (int c = 0; c < 3; ++c)
        cuda_check(cudaMemcpyAsync(u[c], x_.comp(0, c), bytes, cudaMemcpyDeviceToDevice, st), "copy out");
    cuda_check(cudaStreamSynchronize(st), "synchronize");
    return converged;
}

}  // namespace tn
