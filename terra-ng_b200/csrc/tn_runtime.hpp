// Host runtime objects behind the C ABI: device buffers, the per-level device
// mesh, and operator objects.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "tn_boundary.hpp"
#include "tn_grid.hpp"
#include "tn_kernels.hpp"

namespace tn {

// Status codes mirrored from terra_b200.h.
enum Status : int {
    kOk            = 0,
    kErrArg        = -1,
    kErrCuda       = -2,
    kErrAlloc      = -3,
    kErrState      = -4,
    kErrDevice     = -5,
    kErrUnsupported = -6,
    kErrNotConverged = -7,
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw Error(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// Owning device allocation.
class DevBuf {
  public:
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { alloc(bytes); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&)            = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_)
    {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) {
            release();
            p_   = o.p_;
            n_   = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t bytes)
    {
        release();
        if (bytes == 0) return;
        // pad to 256 bytes so 16-byte-rounded bulk reads never leave the allocation
        const size_t padded = (bytes + 255) / 256 * 256;
        if (cudaMalloc(&p_, padded) != cudaSuccess) {
            cudaGetLastError();
            p_ = nullptr;
            throw Error(kErrAlloc, "cudaMalloc of " + std::to_string(padded) + " bytes failed");
        }
        n_ = bytes;
    }
    // alloc unless the buffer already has exactly this size (a rebuild reuses it)
    void ensure(size_t bytes)
    {
        if (p_ == nullptr || n_ != bytes) alloc(bytes);
    }
    void release()
    {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    template <typename T>
    T* as() const
    {
        return static_cast<T*>(p_);
    }
    void*  get() const { return p_; }
    size_t size() const { return n_; }

  private:
    void*  p_ = nullptr;
    size_t n_ = 0;
};

template <typename T>
DevBuf upload(const std::vector<T>& v)
{
    DevBuf b(v.size() * sizeof(T));
    if (!v.empty()) cuda_check(cudaMemcpy(b.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return b;
}

// One mesh level resident on the device (both precisions of the geometry).
struct DeviceLevel {
    ShellLevel host;
    DevBuf     coords64, coords32;  // (10, nl, nl, 3)
    DevBuf     colgeo64, colgeo32;  // (10, nl-1, nl-1, 20) per-column wedge geometry
    DevBuf     radgeo64, radgeo32;  // (nr-1, 3) per-radial-cell factors
    DevBuf     radii64, radii32;    // (nr)
    DevBuf     owned_lat;           // (10, nl, nl) uint8
    DevBuf     dup_offset, dup_members;
    DevBuf     canon_lat;  // (10, nl, nl) int32: lowest lateral index of the node's duplicate class
    IfaceTable iface;
    // linear-transfer weights of this level as the fine level (2 per node), built on first use
    mutable DevBuf linw64, linw32;
    template <typename T>
    const T* linear_weights(cudaStream_t st) const;

    int     nl() const { return host.nl; }
    int     nr() const { return host.nr; }
    int64_t nodes() const { return host.num_stored_nodes(); }
    int64_t cells() const { return 10ll * (host.nl - 1) * (host.nl - 1) * (host.nr - 1); }
    template <typename T>
    const T* coords() const;
    template <typename T>
    const T* radii() const;
    template <typename T>
    const T* colgeo() const;
    template <typename T>
    const T* radgeo() const;
};
template <>
inline const double* DeviceLevel::coords<double>() const
{
    return coords64.as<double>();
}
template <>
inline const float* DeviceLevel::coords<float>() const
{
    return coords32.as<float>();
}
template <>
inline const double* DeviceLevel::colgeo<double>() const
{
    return colgeo64.as<double>();
}
template <>
inline const float* DeviceLevel::colgeo<float>() const
{
    return colgeo32.as<float>();
}
template <>
inline const double* DeviceLevel::radgeo<double>() const
{
    return radgeo64.as<double>();
}
template <>
inline const float* DeviceLevel::radgeo<float>() const
{
    return radgeo32.as<float>();
}
template <>
inline const double* DeviceLevel::radii<double>() const
{
    return radii64.as<double>();
}
template <>
inline const float* DeviceLevel::radii<float>() const
{
    return radii32.as<float>();
}

template <>
const double* DeviceLevel::linear_weights<double>(cudaStream_t st) const;
template <>
const float* DeviceLevel::linear_weights<float>(cudaStream_t st) const;

struct Shell {
    std::vector<std::unique_ptr<DeviceLevel>> levels;  // 0 = coarsest
    DevBuf                                    err;     // device error word
    DevBuf                                    red;     // reduction scratch (partials + result)
    double                                    r_min = 0, r_max = 0;

    const DeviceLevel& level(int l) const
    {
        if (l < 0 || l >= static_cast<int>(levels.size())) throw Error(kErrArg, "level index out of range");
        return *levels[l];
    }
    int* err_word() const { return err.as<int>(); }
};


std::unique_ptr<Shell> make_shell(int lat_level, int rad_level, int num_levels, double r_min, double r_max);

// Operator objects behind tn_operator. Vector arguments are arrays of
// component pointers: velocity = 3 components, pressure = 1, Stokes = 4
// (u_x, u_y, u_z, p). Every apply honours the apply mode (Replace / Add) and the
// communication mode (interface sum of the output or not).
struct Operator {
    const Shell* shell = nullptr;
    int          level = 0;      // velocity (fine) level index
    int          precision = 0;  // 0 f64, 1 f32
    int          apply_mode = 0; // 0 replace, 1 add
    int          comm_mode  = 1; // 1 communicate additively
    int          bc_cmb = 1, bc_surf = 1;

    virtual ~Operator() = default;
    virtual int  src_components() const = 0;
    virtual int  dst_components() const = 0;
    virtual bool dst_on_coarse() const { return false; }
    virtual void apply(void* const* src, void* const* dst, cudaStream_t st) = 0;
    const DeviceLevel& lvl() const { return shell->level(level); }
};

// epsilon-div-div (EpsilonDivDivKerngen). With stored matrices (GCA levels,
// OperatorStoredMatrixMode::Full) the apply runs over the packed element
// matrices instead of the coefficient; boundary conditions are baked into a
// copy of the matrices the first time an apply needs them.
struct EpsDivDivOp : Operator {
    DevBuf k;  // nodal or cell coefficient in `precision` (may be empty in stored mode)
    bool   q0 = false;
    bool   diagonal = false;
    int    tile_y = 0, chunk_x = 0;

    // free slip on both boundaries: the orthonormal rotation modes as coefficients over the raw modes e_i x X
    // (evaluated from the coordinates by the kernels) and the scratch of the penalty dst += eps sum_i (n_i^T src) n_i
    PenaltyCoef pen_coef;
    bool        pen_ready = false;
    DevBuf      pen_scratch;

    bool   stored = false;
    DevBuf mats;              // FP64 unbaked element matrices [342][cells] ([342][sel_count] when selective)
    DevBuf baked64, baked32;  // boundary-baked copies (built lazily; of sel_delta when selective)
    int    baked_bc[2]   = {-1, -1};
    bool   baked32_valid = false;

    // Selective storage (OperatorStoredMatrixMode::Selective, local_matrix_storage.hpp:22-166; the slow path's
    // choice per cell, epsilon_divdiv_kerngen.hpp:1047-1060): GCA matrices on the cells whose coarsest
    // ancestor is marked, the on-the-fly operator of k on all others. mats holds the GCA matrices of the
    // sel_count marked cells (slot s = cell sel_cells[s], sel_slot the inverse map, -1 unmarked); sel_delta
    // holds mats minus the element matrices of k on those cells. The apply is the matrix-free kernel over every
    // cell plus sel_delta (baked) over the slots, which equals the per-cell choice because the boundary
    // treatment and the diagonal mode are linear in the matrix. k32: FP32 copy of k for FP32 applies.
    bool   selective = false;
    bool   sel_built = false;
    int    sel_level_range = 0;
    int    sel_count       = 0;
    DevBuf sel_cells, sel_slot, sel_delta, k32;

    int  src_components() const override { return 3; }
    int  dst_components() const override { return 3; }
    void apply(void* const* src, void* const* dst, cudaStream_t st) override;
    template <typename T>
    void apply_t(const T* const* src, T* const* dst, cudaStream_t st);
    // backward of the apply: grad_cell = d(lambda^T A u)/d log(eta_cell) (Q0 only)
    template <typename T>
    void vjp_logeta(const T* const* u, const T* const* lam, T* grad_cell, cudaStream_t st) const;
    // free-slip/free-slip null-space penalty (epsilon_divdiv_kerngen.hpp:324-445, :711-785)
    bool penalty_active() const { return bc_cmb == 2 && bc_surf == 2; }
    void prepare_penalty(cudaStream_t st);  // orthonormalises the modes (synchronous); no-op unless active or done
    template <typename T>
    void add_penalty(const T* const* src, T* const* dst, cudaStream_t st);
    // stored-matrix helpers
    void ensure_baked(bool need32, cudaStream_t st);
    void set_stored_matrices_from_coefficient(cudaStream_t st);  // element matrices of this level
    int64_t mats_values() const;  // FP64 values of mats
    // selective storage: cells whose ancestor level_range levels down is marked in marks_dev (one byte per cell
    // of that level) get stored matrices once a GCA build fills them (synchronous)
    void set_selective(const uint8_t* marks_dev, int level_range, cudaStream_t st);
    void finish_selective(cudaStream_t st);  // after the build: the correction sel_delta
    void materialize_full(cudaStream_t st);  // selective -> full storage (unmarked cells get element matrices)
    // the matrix of every cell (stored, GCA or element matrix) into out [342][cells], unbaked
    void effective_matrices(DevBuf& out, cudaStream_t st) const;
    // FP32 applies of an FP64 operator: FP32 coefficient and the penalty set-up (synchronous, before capture)
    void prepare_fp32(cudaStream_t st);
};
// TwoGridGCA (gca.hpp:41-531): coarse.mats = sum P^T A_fine P with A_fine the
// fine operator's stored matrices or its on-the-fly Neumann element matrices.
// linear: InterpolationMode::Linear (the fine level's linear-transfer weights) instead of Constant.
void gca_coarsen(const EpsDivDivOp& fine, EpsDivDivOp& coarse, cudaStream_t st, bool linear = false,
                 bool tensor_cores = true);

// B (DivergenceKerngen): velocity level -> pressure level (level - 1).
struct DivergenceOp : Operator {
    mutable DevBuf scratch;  // one value per fine wedge
    int  src_components() const override { return 3; }
    int  dst_components() const override { return 1; }
    bool dst_on_coarse() const override { return true; }
    void apply(void* const* src, void* const* dst, cudaStream_t st) override;
    template <typename T>
    void apply_t(const T* const* src, T* p, cudaStream_t st) const;
};

// B^T (GradientKerngen): pressure level -> velocity level.
struct GradientOp : Operator {
    mutable DevBuf scratch;  // one value per fine wedge
    int  src_components() const override { return 1; }
    int  dst_components() const override { return 3; }
    void apply(void* const* src, void* const* dst, cudaStream_t st) override;
    template <typename T>
    void apply_t(const T* p, T* const* dst, cudaStream_t st) const;
};

// [A B^T; B 0] (EpsDivDivStokes, epsilon_divdiv_stokes.hpp:55-84).
struct StokesOp : Operator {
    EpsDivDivOp  A;
    GradientOp   BT;
    DivergenceOp B;
    int          src_components() const override { return 4; }
    int          dst_components() const override { return 4; }
    void         apply(void* const* src, void* const* dst, cudaStream_t st) override;
};

template <typename T>
void zero_components(int64_t n, int ncomp, T* const* v, cudaStream_t st);

// XDMF output / checkpoint in the reference's format (xdmf.cpp)
struct Xdmf;
Xdmf* xdmf_create(const Shell* sh, int level, const std::string& dir, int geometry_bytes);
void  xdmf_add(Xdmf* x, const std::string& name, int precision, int ncomp, void* const* comps, int out_bytes);
void  xdmf_write(Xdmf* x);
void  xdmf_destroy(Xdmf* x);
void  xdmf_read(const Shell* sh, int level, const std::string& dir, const std::string& name, int step, int precision,
                int ncomp, void* const* comps);

}  // namespace tn
