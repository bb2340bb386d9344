/*
 * Stub bodies for the CGNS stand-in header (test oracle only).  Any call is a
 * configuration error of the oracle driver: it must select CSV output and a
 * Cartesian or gmsh mesh.  The stubs therefore fail loudly.
 */
#include <stdio.h>
#include <stdlib.h>

#include "cgnslib.h"

static int cgns_unavailable(const char *name)
{
	fprintf(stderr, "oracle: CGNS call %s reached; CGNS I/O is not built "
		"into the oracle\n", name);
	exit(3);
	return 1;
}

void cg_error_exit(void) { cgns_unavailable("cg_error_exit"); }
void cg_free() { cgns_unavailable("cg_free"); }
int cg_open() { return cgns_unavailable("cg_open"); }
int cg_close() { return cgns_unavailable("cg_close"); }
int cg_goto() { return cgns_unavailable("cg_goto"); }
int cg_base_write() { return cgns_unavailable("cg_base_write"); }
int cg_zone_write() { return cgns_unavailable("cg_zone_write"); }
int cg_zone_read() { return cgns_unavailable("cg_zone_read"); }
int cg_coord_write() { return cgns_unavailable("cg_coord_write"); }
int cg_coord_read() { return cgns_unavailable("cg_coord_read"); }
int cg_section_write() { return cgns_unavailable("cg_section_write"); }
int cg_section_read() { return cgns_unavailable("cg_section_read"); }
int cg_nsections() { return cgns_unavailable("cg_nsections"); }
int cg_elements_read() { return cgns_unavailable("cg_elements_read"); }
int cg_sol_write() { return cgns_unavailable("cg_sol_write"); }
int cg_field_write() { return cgns_unavailable("cg_field_write"); }
int cg_field_read() { return cgns_unavailable("cg_field_read"); }
int cg_link_write() { return cgns_unavailable("cg_link_write"); }
int cg_array_write() { return cgns_unavailable("cg_array_write"); }
int cg_biter_write() { return cgns_unavailable("cg_biter_write"); }
int cg_ziter_write() { return cgns_unavailable("cg_ziter_write"); }
int cg_descriptor_write() { return cgns_unavailable("cg_descriptor_write"); }
int cg_descriptor_read() { return cgns_unavailable("cg_descriptor_read"); }
int cg_nbocos() { return cgns_unavailable("cg_nbocos"); }
int cg_boco_info() { return cgns_unavailable("cg_boco_info"); }
int cg_boco_write() { return cgns_unavailable("cg_boco_write"); }
int cg_grid_write() { return cgns_unavailable("cg_grid_write"); }
int cg_ElementDataSize() { return cgns_unavailable("cg_ElementDataSize"); }
