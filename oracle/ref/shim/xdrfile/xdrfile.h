/* Empty stand-in for the xdrfile library headers: the reference classes built
   here only declare, never call, their trajectory readers. */
#pragma once
