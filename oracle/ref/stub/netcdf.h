/* Empty stand-in: the reference's kernel files include netcdf.h but use none
 * of it (test infrastructure). */
#pragma once
