/*
 * Test infrastructure only: entry points of DAAL's data-management and
 * environment layers that the dense Lloyd kernel links against but never
 * calls (model serialization, the object factory, CPU-feature queries).
 * They abort if reached, so an unexpected call cannot pass silently.
 */
#include "data_management/data/homogen_numeric_table.h"
#include "data_management/data/factory.h"
#include "services/env_detect.h"

#include <cstdlib>

namespace daal { namespace data_management { namespace interface1 {
void SerializationIface::serialize(InputDataArchive &)
{
    std::abort();
}
Factory & Factory::instance()
{
    std::abort();
}
SerializationIface * Factory::createObject(int)
{
    std::abort();
}
}}} // namespace daal::data_management::interface1

namespace daal { namespace services { namespace interface1 {
Environment * Environment::getInstance()
{
    return nullptr;
}
int Environment::getCpuId(int)
{
    return 0;
}
}}} // namespace daal::services::interface1
