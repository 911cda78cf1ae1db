"""braidlab call surface for the B200 packer.

The reference's orchestration package drives its engines through
``braidlab.engine`` (binary names, argv, ``done:`` parsing), ``braidlab.config``
(``Job`` / ``Campaign``) and reads frames with ``braidlab.frames``.  This package
keeps those interfaces -- same names, arguments, identities and errors -- so the
reference's callers can launch the B200 packer (``universe-generator_b200/bin``)
in place of the CUDA engines.  It contains no compute: the packer is libug.so.
"""
