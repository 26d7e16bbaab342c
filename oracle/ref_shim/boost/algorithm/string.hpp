/* Empty stand-in: the hot-path translation units of the reference include this
   header through mhd2d.hpp but use nothing from it. */
#pragma once
