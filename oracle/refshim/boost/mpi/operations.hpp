// FieldPatch.hh includes this for its MPI reduction operator; one process here.
#pragma once
