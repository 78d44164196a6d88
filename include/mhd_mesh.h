/* Host-side mesh services of the caller: the signed cell complex, its metric and its
 * boundary classification, in exactly the layout the reference's uns::CellComplex,
 * uns::Geometry and mhd::BoundaryInfo hold (signed CSR: int64 ptr, int32 idx, int8 sgn;
 * Vec3 arrays as 3 doubles per entity).  These are the inputs of the device hot path
 * (mhd_gpu.h); in a reference build they come from the reference itself, here they are
 * produced natively so the library runs stand-alone.
 *
 * Numbering, orientation and classification follow the reference bit for bit:
 *   builder      include/uns/complex/ComplexBuilder.h:14-41, src/uns/complex/ComplexBuilder.cpp:20-134
 *   generators   src/uns/generate/BoxMesh.cpp:5-33, CubedSphereMesh.cpp:12-83, HexMesh.cpp:7-18
 *   geometry     src/uns/geometry/Geometry.cpp:17-169 (+ check_geometry :171-205)
 *   boundary     Common/boundary/BoundaryInfo.cpp:9-49
 *   hash         src/uns/complex/CellComplex.cpp:56-70 (uns::topology_hash)
 * The 6-tetrahedron split of hexahedral meshes (mhdm_split_tets) has no counterpart in the
 * reference, which generates hexahedra only; it feeds tetrahedra to the same builder.
 *
 * Every function returns 0 on success and a negative status on error; the message of the
 * last error of the calling thread is returned by mhdm_last_error(). */
#ifndef MHD_MESH_H
#define MHD_MESH_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct MhdHostMesh MhdHostMesh;

const char *mhdm_last_error(void);

/* Generic polyhedral cells (reference ComplexBuilder::add_cell + tag_face + finish).  Cell c
 * owns the outward face loops cell_ptr[c] .. cell_ptr[c+1]-1; loop l has the nodes
 * loop_nodes[loop_ptr[l] .. loop_ptr[l+1]-1] counter-clockwise seen from outside.  Tagged face
 * t has the nodes tag_nodes[tag_ptr[t] .. tag_ptr[t+1]-1] in any order and the tag id tag_id[t];
 * tag_names (n_names strings, [0] unused) name the tag ids. */
int mhdm_from_cells(int32_t n_nodes, const double *x, int32_t n_cells, const int64_t *cell_ptr, const int64_t *loop_ptr,
                    const int32_t *loop_nodes, const int32_t *material, int32_t n_tagged, const int64_t *tag_ptr,
                    const int32_t *tag_nodes, const int32_t *tag_id, int32_t n_names, const char *const *tag_names,
                    MhdHostMesh **out);

/* Hexahedral generators (reference uns::make_box / make_cubed_sphere_shell + build_mesh).
 * as_tets != 0 cuts every hexahedron into the 6 tetrahedra of its lattice body diagonal
 * (Kuhn split: corner 0 -> corner 7 of the reference's local node order) before building;
 * jitter > 0 moves every node not on the domain boundary by jitter*h uniformly in each
 * coordinate (box only; h = cell size per axis) with the splitmix64 stream of `seed`. */
int mhdm_box(int32_t nx, int32_t ny, int32_t nz, const double *lo, const double *hi, int32_t as_tets, double jitter,
             uint64_t seed, MhdHostMesh **out);
int mhdm_shell(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch, int32_t as_tets,
               MhdHostMesh **out);

/* The shell's hexahedral list alone, for a complex built elsewhere (mhd_gpu_tet_build): nodes and tag
 * names as mhdm_shell makes them, and the arrays "hex" (8 nodes per hexahedron, the reference's local
 * corner order), "hex_material", "tag_tri" (3 nodes per tagged triangle of the tetrahedral split, in the
 * order mhdm_shell tags them) and "tag_tri_id"; no complex yet (counts: nodes only). */
int mhdm_shell_hexes(int32_t ncube, int32_t nr, int32_t n_solid, double r_in, double r_out, double r_stretch, MhdHostMesh **out);
/* Size the complex of such a mesh (faces_per_cell entries per c2f row, edges_per_face per f2e row, 2 per
 * e2n row; the upward tables likewise) for the caller to fill through mhdm_array_mut; drops the hexahedral
 * list and any geometry or boundary classification. */
int mhdm_reserve_complex(MhdHostMesh *m, int64_t n_edges, int64_t n_faces, int64_t n_cells, int32_t faces_per_cell,
                         int32_t edges_per_face);
/* mhdm_array with a writable pointer */
void *mhdm_array_mut(MhdHostMesh *m, const char *name, int64_t *count);

/* The same complex built again with its cells in the given order (new cell i = old cell order[i]):
 * faces and edges are numbered in creation order of the new cell sequence, tags and materials carried
 * over, geometry not computed.  With a locality order (HostMesh.locality_order: Morton order of the cell
 * centres) this is the locality renumbering of a mesh that arrives in an arbitrary order; reordering by
 * the inverse permutation rebuilds the original numbering exactly (same uns::topology_hash). */
int mhdm_reorder_cells(const MhdHostMesh *m, const int32_t *order, MhdHostMesh **out);

void mhdm_free(MhdHostMesh *m);

/* counts[0..3] = nodes, edges, faces, cells */
void mhdm_counts(const MhdHostMesh *m, int32_t *counts);
uint64_t mhdm_topology_hash(const MhdHostMesh *m);

/* uns::compute_geometry on this mesh (idempotent). */
int mhdm_compute_geometry(MhdHostMesh *m);
/* mhd::BoundaryInfo::build: bc_default and per-tag-name types ("wall", "inflow", "outflow",
 * "farfield"); u_inf decides farfield faces. */
int mhdm_boundary(MhdHostMesh *m, const char *bc_default, int32_t n_pairs, const char *const *tag_names,
                  const char *const *types, const double *u_inf);
/* The per-tag-id boundary types that mhdm_boundary would apply (for mhd_gpu_boundary): tag_type[t] for the
 * mesh's tag ids t < n_tags (cap entries available), type_none for tag 0 and unknown ids; codes 1 wall,
 * 2 inflow, 3 outflow, 5 farfield, 0 unknown type name. */
int mhdm_tag_types(const MhdHostMesh *m, const char *bc_default, int32_t n_pairs, const char *const *tag_names,
                   const char *const *types, int32_t cap, int8_t *tag_type, int8_t *type_none, int32_t *n_tags);
/* Install a boundary classification computed elsewhere (face kinds and edge modes, one per face / edge). */
int mhdm_set_boundary(MhdHostMesh *m, const int8_t *face_kind, const int8_t *edge_mode);

/* Pointer to the named array and its element count (NULL / -1 if unknown or not computed).
 * Names: x, e2n_ptr/idx/sgn, f2e_*, c2f_*, e2f_*, f2c_*, cell_material, face_tag, edge_vec,
 * edge_mid, edge_len, face_area, face_center, face_area_mag, cell_center, cell_volume,
 * cell_min_tet_volume, edge_dual_area, ec_ptr, ec_cell, ec_weight, ef_weight, ec_misoriented,
 * star0..star3, face_kind, edge_mode.  The pointer stays valid until mhdm_free. */
const void *mhdm_array(const MhdHostMesh *m, const char *name, int64_t *count);

/* Install a geometry computed elsewhere (mhd_gpu_compute_geometry) in place of mhdm_compute_geometry's:
 * the arrays are copied (sizes as in MhdGeometryArgs; ec lists of ec_ptr[n_edges] entries). */
typedef struct MhdGeometryArrays {
    const double *edge_vec, *edge_mid, *edge_len, *face_area, *face_center, *face_area_mag, *cell_center, *cell_volume,
        *cell_min_tet_volume, *edge_dual_area, *ec_weight, *ef_weight, *star0, *star1, *star2, *star3;
    const int64_t *ec_ptr;
    const int32_t *ec_cell, *ec_misoriented;
} MhdGeometryArrays;
int mhdm_set_geometry(MhdHostMesh *m, const MhdGeometryArrays *g);

/* ------------------------------------------------------------------ UNSBIN field files
 * uns::io::write_fields / read_fields (src/uns/io/MeshIO.cpp:117-150) over the UNSBIN container of
 * src/uns/io/BinContainer.cpp (little endian: magic "UNSBIN\0\1", u64 record count, records of u32 name
 * length | name | u8 dtype | 3 pad bytes | u32 cols | u64 rows | payload padded to 8 bytes).  The files are
 * the reference's restart / coarse-solution files (docs/FileFormats.md, "Coarse / restart solution").
 * dims: uns::Dim (0 node, 1 edge, 2 face, 3 cell); values[i] holds counts[i] doubles (entities x ncomp). */
int mhdm_write_fields(const char *path, uint64_t topology_hash, int32_t n, const char *const *names, const int32_t *dims,
                      const int32_t *ncomps, const int64_t *counts, const double *const *values);
typedef struct MhdFieldFile MhdFieldFile;
/* read a field file; the records come in the order of its index */
int mhdm_read_fields(const char *path, MhdFieldFile **out);
void mhdm_fields_free(MhdFieldFile *f);
/* record count and the stored topology hash */
int32_t mhdm_fields_count(const MhdFieldFile *f, uint64_t *topology_hash);
/* record i: name (len bytes incl. the terminator), dim, ncomp, value count; values copied when out != NULL */
int mhdm_field(const MhdFieldFile *f, int32_t i, char *name, int32_t len, int32_t *dim, int32_t *ncomp, int64_t *count, double *out);

#ifdef __cplusplus
}
#endif
#endif
