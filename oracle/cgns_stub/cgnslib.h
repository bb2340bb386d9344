/*
 * Minimal stand-in for the CGNS library header, used only to compile the
 * reference ccfd sources as a CPU test oracle without building CGNS
 * (a cmake project).  CGNS is file I/O only in ccfd; none of its arithmetic
 * is on the residual-and-update path.  Every function here is a stub that
 * reports an error: the oracle driver selects CSV output and the Cartesian /
 * gmsh mesh readers, so no CGNS call is ever reached.
 *
 * Names and enum members follow the public CGNS 4.x API so that the
 * reference sources compile unchanged; signatures are left unspecified
 * (K&R-style declarations) because the stubs never run.
 */
#ifndef CCFD_ORACLE_CGNS_STUB_H
#define CCFD_ORACLE_CGNS_STUB_H

typedef long cgsize_t;

typedef enum { DataTypeNull, DataTypeUserDefined, Integer, RealSingle,
	       RealDouble, Character, LongInteger } DataType_t;
typedef enum { ZoneTypeNull, ZoneTypeUserDefined, Structured,
	       Unstructured } ZoneType_t;
typedef enum { GridLocationNull, GridLocationUserDefined, Vertex, CellCenter,
	       FaceCenter, IFaceCenter, JFaceCenter, KFaceCenter,
	       EdgeCenter } GridLocation_t;
typedef enum { ElementTypeNull, ElementTypeUserDefined, NODE, BAR_2, BAR_3,
	       TRI_3, TRI_6, QUAD_4, QUAD_8, QUAD_9, TETRA_4, TETRA_10,
	       PYRA_5, PYRA_14, PENTA_6, PENTA_15, PENTA_18, HEXA_8, HEXA_20,
	       HEXA_27, MIXED } ElementType_t;
typedef enum { PointSetTypeNull, PointSetTypeUserDefined, PointList,
	       PointListDonor, PointRange, PointRangeDonor, ElementRange,
	       ElementList, CellListDonor } PointSetType_t;
typedef enum { BCTypeNull, BCTypeUserDefined, BCAxisymmetricWedge, BCDegenerateLine,
	       BCDegeneratePoint, BCDirichlet, BCExtrapolate, BCFarfield,
	       BCGeneral } BCType_t;

#define CG_MODE_READ 0
#define CG_MODE_WRITE 1
#define CG_MODE_MODIFY 2

void cg_error_exit(void);
void cg_free();
int cg_open();
int cg_close();
int cg_goto();
int cg_base_write();
int cg_zone_write();
int cg_zone_read();
int cg_coord_write();
int cg_coord_read();
int cg_section_write();
int cg_section_read();
int cg_nsections();
int cg_elements_read();
int cg_sol_write();
int cg_field_write();
int cg_field_read();
int cg_link_write();
int cg_array_write();
int cg_biter_write();
int cg_ziter_write();
int cg_descriptor_write();
int cg_descriptor_read();
int cg_nbocos();
int cg_boco_info();
int cg_boco_write();
int cg_grid_write();
int cg_ElementDataSize();

#endif
