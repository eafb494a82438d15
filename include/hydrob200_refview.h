/*
 * hydrob200_refview.h -- drop-in entry points over the reference's own device
 * arrays (caller-owned, reference layout, updated in place).
 *
 * hb_ref_mesh_view has the memory layout of the reference's MeshView
 * (cuda_native_impl/hydro-cal-src/include/mesh/mesh.hpp:114-141 with
 * CellView cell.hpp:28-61 and SideView side.hpp:29-52) for Real = double;
 * hb_ref_mesh_view_f32 that of the fp32 tree (Real = float,
 * cuda_native_impl/fp32_src/hydro-cal-src/include/common.hpp:15).
 *
 * The C++ overloads at the end have the exact signatures of the reference's
 * functors.cuh:59-65 (functors.cu:787-818), so a program built against the
 * reference headers links against this library in place of functors.cu.
 */
#ifndef HYDROB200_REFVIEW_H
#define HYDROB200_REFVIEW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hb_ref_cell_view {
    double *H, *U, *V, *W, *Z;
    const int32_t *NHQ1;
    const double *ZBC, *ZB1, *AREA, *FNC, *BoundaryFeature;
    const double *ZW, *QW, *QT, *DQT, *ZT, *DZT;
} hb_ref_cell_view;

typedef struct hb_ref_side_view {
    double *KLAS;
    const double *NAC, *SIDE, *COSF, *SINF, *SLCOS, *SLSIN;
    double *FLUX0, *FLUX1, *FLUX2, *FLUX3;
} hb_ref_side_view;

typedef struct hb_ref_mesh_view {
    int32_t NHQ, NQ, NZ, NWE, NDAYS, CELL;
    double DT, HM1, HM2, JL;
    hb_ref_cell_view cells;
    hb_ref_side_view sides;
} hb_ref_mesh_view;

typedef struct hb_ref_cell_view_f32 {
    float *H, *U, *V, *W, *Z;
    const int32_t *NHQ1;
    const float *ZBC, *ZB1, *AREA, *FNC, *BoundaryFeature;
    const float *ZW, *QW, *QT, *DQT, *ZT, *DZT;
} hb_ref_cell_view_f32;

typedef struct hb_ref_side_view_f32 {
    float *KLAS;
    const float *NAC, *SIDE, *COSF, *SINF, *SLCOS, *SLSIN;
    float *FLUX0, *FLUX1, *FLUX2, *FLUX3;
} hb_ref_side_view_f32;

typedef struct hb_ref_mesh_view_f32 {
    int32_t NHQ, NQ, NZ, NWE, NDAYS, CELL;
    float DT, HM1, HM2, JL;
    hb_ref_cell_view_f32 cells;
    hb_ref_side_view_f32 sides;
} hb_ref_mesh_view_f32;

/* CalculateFlux(mesh, kt, jt, stream), functors.cu:787-792: fluxes of every
 * slot of day jt, step kt, into sides.FLUX0..3 (and KLAS 7 -> 0 on breach).
 * `variant` is hb_variant; `stream` a cudaStream_t. Asynchronous. */
int hb_ref_calculate_flux(const hb_ref_mesh_view *mesh, int32_t kt, int32_t jt, int32_t variant, void *stream);
/* UpdateCell(mesh, stream), functors.cu:794-799: H, U, V, Z, W in place. */
int hb_ref_update_cell(const hb_ref_mesh_view *mesh, int32_t variant, void *stream);
int hb_ref_calculate_flux_f32(const hb_ref_mesh_view_f32 *mesh, int32_t kt, int32_t jt, int32_t variant, void *stream);
int hb_ref_update_cell_f32(const hb_ref_mesh_view_f32 *mesh, int32_t variant, void *stream);
/* Bits of hb_status codes raised by these kernels since the last call (then cleared). */
int hb_ref_take_device_errors(uint32_t *bits);

/* One whole timestep (CalculateFlux then UpdateCell, fp64) over the caller's
 * reference-layout arrays that allocates no device memory at all.  This entry
 * point has no counterpart in the reference.
 *
 * It is meant for callers that cannot call cudaMalloc: a host framework that
 * owns the device allocator (a caching allocator that must see every byte), a
 * program whose memory budget is fixed when it starts, or code running where
 * an allocation would synchronise or fail.  The scratch that carries each
 * slot's terms of the cell sums from the flux pass to the update pass lives in
 * a fixed array inside the library instead, HB_REF_STEP_STATIC_MAX_CELLS cells
 * (8 MiB), which every GPU that loads the library holds until the process
 * exits.
 *
 * - Meshes with more cells are rejected with HB_E_TOO_LARGE before anything is
 *   launched.
 * - The first call on a device looks up the array's device address
 *   (cudaGetSymbolAddress) with that device current; make that first call
 *   before any stream capture.  The address is kept for the life of the
 *   process, so do not use this entry point on a device after
 *   cudaDeviceReset (or any other teardown of its primary context): the
 *   module, and with it the array, is loaded anew there and the kept address
 *   no longer points at it.
 * - Every call shares the one array: calls whose work overlaps on the GPU
 *   (other streams, other threads) race on it.  Each call writes every term it
 *   later reads, so nothing needs clearing between calls.
 * - Results are bit-identical to hb_ref_calculate_flux followed by
 *   hb_ref_update_cell: state updated in place, FLUX0..3 and KLAS written as
 *   CalculateFlux writes them. */
#define HB_REF_STEP_STATIC_MAX_CELLS 65536
int hb_ref_step_static(const hb_ref_mesh_view *mesh, int32_t kt, int32_t jt, int32_t variant, void *stream);

#ifdef __cplusplus
}  /* extern "C" */

/* Reference-signature overloads (functors.cuh:59-65), variant H.  MeshView is
 * the reference's own type; only its layout is relied upon. */
struct MeshView;
struct CUstream_st;
void CalculateFlux(const MeshView &mesh, int kt, int jt, CUstream_st *stream);
void UpdateCell(const MeshView &mesh, CUstream_st *stream);
void CalculateFlux(const MeshView &mesh, int kt, int jt);
void UpdateCell(const MeshView &mesh);
#endif

#endif
