/* sg_enum.cpp -- host entry of the error-pattern order builder (sg_enum.h). */
#include "sg_enum.h"

extern "C" size_t sg_enum_build(int32_t ic, uint32_t* out)
{
    return sg_enum_build_impl(ic, out);
}
